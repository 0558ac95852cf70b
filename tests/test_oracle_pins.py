"""The CPU oracle pinned against the reference's own fixtures (no GPU).

Fixtures in tests/golden/ were extracted from the reference checkout by
tests/golden/make_golden.py.
"""
import json
import os

import numpy as np
import pytest
from scipy.special import hankel1

from conftest import GOLDEN, golden
from cugmres_b200 import problems as P


@pytest.mark.parametrize("N", [32, 64])
def test_green_block_matches_G_prep(oracle, N):
    gp = golden(f"ref_G_prep_{N}.npz")["g_prep"].astype(np.complex128)
    og = oracle.green_block_reference(N, True)
    # G_prep is written with ~8 significant digits
    assert np.abs(gp[:N, :N] - og).max() < 3e-7
    M = 2 * N - 1
    idx = np.arange(M)
    d = np.where(idx < N, idx, M - idx)
    full = og[d[:, None], d[None, :]]
    assert np.abs(full - gp).max() < 3e-7


@pytest.mark.parametrize("N", [32, 64, 256])
def test_cylinder_masks(N):
    d = golden(f"ref_cylinder_{N}.npz")
    m = np.unpackbits(d["mask"])[: N * N].reshape(N, N).astype(bool)
    assert (m == P.cylinder_mask(N)).all()


@pytest.mark.parametrize("N", [8, 16, 32])
def test_oracle_matvec_matches_pygmres(oracle, N):
    d = golden("pygmres_matvec.npz")
    x, eps, k, y = d[f"x_{N}"], d[f"eps_{N}"], float(d[f"k_{N}"]), d[f"y_{N}"]
    gb = d[f"green_block_{N}"]
    gh = oracle.spectrum(gb, 2 * N)
    yo = oracle.matvec(gh, (k * k * eps).reshape(N, N), x.reshape(N, N)).ravel()
    # the reference pads into a complex64 array (PyGMRES/GMRES.py:37), hence ~1e-7
    assert np.abs(yo - y).max() / np.abs(y).max() < 2e-7


@pytest.mark.parametrize("N", [8, 16, 32])
def test_oracle_transpose_matches_reference_pygmres(oracle, N):
    """The reference's own matvec(x, eps, k, transpose=True) = x - chi G x."""
    d = golden("pygmres_matvec.npz")
    x, eps, k, yt = d[f"x_{N}"], d[f"eps_{N}"], float(d[f"k_{N}"]), d[f"yt_{N}"]
    gh = oracle.spectrum(d[f"green_block_{N}"], 2 * N)
    yo = oracle.matvec_transpose(gh, (k * k * eps).reshape(N, N), x.reshape(N, N)).ravel()
    assert np.abs(yo - yt).max() / np.abs(yt).max() < 2e-7


def test_oracle_fft_matches_numpy(oracle):
    rng = np.random.default_rng(0)
    for L in (8, 16, 12, 48, 64):
        a = rng.standard_normal((L, L)) + 1j * rng.standard_normal((L, L))
        f = oracle.fft2d(a, -1)
        assert np.abs(f - np.fft.fft2(a)).max() < 1e-12 * L * L
        b = oracle.fft2d(a, +1)
        assert np.abs(b - np.fft.ifft2(a) * L * L).max() < 1e-12 * L * L


def test_oracle_matvec_matches_dense_bttb(oracle):
    N = 8
    rng = np.random.default_rng(1)
    g = oracle.green_block_helmholtz(N, 2 * np.pi, 0.05)
    chi = rng.random((N, N))
    x = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    for L in (2 * N, 2 * N + 4, 32):
        y = oracle.matvec(oracle.spectrum(g, L), chi, x)
        i, j = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
        I, J = i.ravel(), j.ravel()
        G = g[np.abs(I[:, None] - I[None, :]), np.abs(J[:, None] - J[None, :])]
        yd = x.ravel() - G @ (chi.ravel() * x.ravel())
        assert np.abs(y.ravel() - yd).max() < 1e-13


def test_mkl_solution_256(oracle):
    """FFT_GMRES_with_MKL for N=256, maxiter=44, x0 = b = plane wave
    (MKL_GMRES_test_09122019/source/main.cpp:16-56) against its saved output."""
    N = 256
    d = golden("ref_mkl_solution_256_m44.npz")
    ref = d["solution"].astype(np.complex128)
    pr = P.reference_cylinder(N)
    gh = oracle.spectrum(oracle.green_block_reference(N, True), 2 * N)
    x, res, n, flag, info = oracle.gmres_reference(gh, pr["chi"], pr["b"], pr["x0"], 44, 1e-8)
    assert n == 44 and info == 0
    assert abs(res[0] - 518.983) < 1e-2
    # the MKL run is single precision: agreement to ~1e-5 is all it can pin
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 3e-5
    x32, res32, n32, flag32, _ = oracle.gmres_reference(
        gh.astype(np.complex64), pr["chi"].astype(np.float32), pr["b"].astype(np.complex64),
        pr["x0"].astype(np.complex64), 44, 1e-8, precision="c64")
    assert np.linalg.norm(x32 - ref) / np.linalg.norm(ref) < 6e-5
    # single-precision residual estimate of the same order as the MKL run's 4.0055e-4
    assert 1e-4 < res32[-1] < 2e-3 and 1e-4 < float(d["residual_estimate"]) < 2e-3
    # the complex128 restatement converges much further (true residual)
    r = oracle.matvec(gh, pr["chi"], x, b=pr["b"])
    assert np.linalg.norm(r) < 1e-8
    # Mie-series plateau published in Results/relative_errors_256_0.npy
    an = golden("ref_analytical_256.npz")["field"].astype(np.complex128)
    pub = json.load(open(os.path.join(GOLDEN, "ref_results.json")))["relative_errors_256"][-1]
    assert abs(np.linalg.norm(x - an) / np.linalg.norm(an) - pub) < 1e-4


def test_helmholtz_green_block_matches_scipy(oracle):
    N, k0, h = 12, 2 * np.pi, 0.05
    g = P.green_block("helmholtz", N, k0, h)
    i, j = np.mgrid[:N, :N]
    r = h * np.sqrt(i ** 2 + j ** 2.0)
    ref = np.zeros((N, N), complex)
    ref[r > 0] = 0.25j * hankel1(0, k0 * r[r > 0]) * h * h
    a = h / np.sqrt(np.pi)
    ref[0, 0] = (1j * np.pi * a / (2 * k0)) * hankel1(1, k0 * a) - 1 / k0 ** 2
    assert np.abs(g - ref).max() / np.abs(ref).max() < 1e-13
    assert np.abs(oracle.green_block_helmholtz(N, k0, h) - g).max() < 1e-15


def _dense_operator(g, c):
    N = g.shape[0]
    i, j = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    I, J = i.ravel(), j.ravel()
    G = g[np.abs(I[:, None] - I[None, :]), np.abs(J[:, None] - J[None, :])]
    return np.eye(N * N) - G * c.ravel()[None, :]


@pytest.mark.parametrize("ortho", ["mgs", "cgs2"])
def test_oracle_gmres_matches_dense_solve(oracle, ortho):
    pr = P.helmholtz(16, 2.25, seed=3)
    gh = oracle.spectrum(pr["g_block"], 32)
    c = pr["chi"] * pr["chi_scale"]
    out = oracle.gmres(gh, c, pr["b"], restart=30, maxiter=300, tol=1e-12, ortho=ortho)
    assert out["status"] == 0 and out["true_res"] <= 1e-12
    xd = np.linalg.solve(_dense_operator(pr["g_block"], c), pr["b"].ravel()).reshape(16, 16)
    assert np.linalg.norm(out["x"] - xd) / np.linalg.norm(xd) < 1e-10


def test_oracle_rotation_formulas_share_the_residual_estimate(oracle):
    pr = P.helmholtz(16, 2.25, seed=4)
    gh = oracle.spectrum(pr["g_block"], 32)
    c = pr["chi"] * pr["chi_scale"]
    a = oracle.gmres(gh, c, pr["b"], restart=40, maxiter=40, tol=0.0, rotation="unitary")
    b = oracle.gmres(gh, c, pr["b"], restart=40, maxiter=40, tol=0.0, rotation="reference")
    assert np.allclose(a["res_hist"], b["res_hist"], rtol=1e-8, atol=1e-14)


def test_oracle_mixed_precision_refinement(oracle):
    pr = P.helmholtz(32, 2.25, seed=5)
    gh = oracle.spectrum(pr["g_block"], 64)
    c = pr["chi"] * pr["chi_scale"]
    ir = oracle.gmres_ir(gh, c, pr["b"], inner_restart=20, inner_tol=1e-5, tol=1e-10)
    ref = oracle.gmres(gh, c, pr["b"], restart=200, maxiter=2000, tol=1e-13)
    assert ir["status"] == 0 and ir["true_res"] <= 1e-10
    assert np.linalg.norm(ir["x"] - ref["x"]) / np.linalg.norm(ref["x"]) < 1e-8
