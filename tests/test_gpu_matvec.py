"""GPU matvec (fused Stockham FFT passes) against the CPU oracle and the
reference's NumPy matvec, through the C-ABI."""
import numpy as np
import pytest

from conftest import golden
import cugmres_b200 as cg
from cugmres_b200 import problems as P

pytestmark = pytest.mark.gpu


def _rand(N, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))


@pytest.mark.parametrize("N", [2, 5, 8, 16, 33, 64, 100, 128, 256, 512])
def test_matvec_fp64_vs_oracle(solver, oracle, N):
    pr = P.helmholtz(N, 4.0, seed=N)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = _rand(N, 7)
    y = solver.matvec(x)
    gh = oracle.spectrum(pr["g_block"], solver.L)
    yo = oracle.matvec(gh, pr["chi"] * pr["chi_scale"], x)
    assert np.abs(y - yo).max() / np.abs(yo).max() < 1e-13


@pytest.mark.parametrize("N", [16, 64, 256, 1024])
def test_matvec_fp32_vs_oracle(solver, oracle, N):
    pr = P.helmholtz(N, 2.25, seed=1)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = _rand(N, 3).astype(np.complex64)
    y = solver.matvec(x, precision="fp32")
    assert y.dtype == np.complex64
    gh = oracle.spectrum(pr["g_block"], solver.L)
    yo = oracle.matvec(gh, pr["chi"] * pr["chi_scale"], x.astype(np.complex128))
    assert np.abs(y - yo).max() / np.abs(yo).max() < 2e-6


def test_matvec_matches_dense_bttb(solver):
    N = 12
    pr = P.helmholtz(N, 3.0, seed=2)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = _rand(N, 4)
    y = solver.matvec(x)
    g = pr["g_block"]
    i, j = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    I, J = i.ravel(), j.ravel()
    G = g[np.abs(I[:, None] - I[None, :]), np.abs(J[:, None] - J[None, :])]
    yd = x.ravel() - G @ (pr["chi"].ravel() * pr["chi_scale"] * x.ravel())
    assert np.abs(y.ravel() - yd).max() / np.abs(yd).max() < 1e-13


@pytest.mark.parametrize("N", [8, 16, 32])
def test_pygmres_matvec_golden(cuda_device, N):
    d = golden("pygmres_matvec.npz")
    x, eps, k, y = d[f"x_{N}"], d[f"eps_{N}"], float(d[f"k_{N}"]), d[f"y_{N}"]
    out = cg.matvec(x, eps, k, device=cuda_device)
    assert out.shape == (N * N, 1)
    assert np.abs(out.ravel() - y).max() / np.abs(y).max() < 2e-7
    blk, G = cg.matvec(x, eps, k, qweq=True)
    assert np.abs(G - d[f"toeplitz_{N}"]).max() < 1e-15


def test_operator_from_G_prep(solver, oracle):
    N = 64
    gp = golden("ref_G_prep_64.npz")["g_prep"]
    pr = P.reference_cylinder(N)
    solver.set_operator_circulant(gp, pr["chi"], 1.0)
    x = _rand(N, 9)
    y = solver.matvec(x)
    gh = oracle.spectrum(gp[:N, :N].astype(np.complex128), solver.L)
    yo = oracle.matvec(gh, pr["chi"], x)
    assert np.abs(y - yo).max() / np.abs(yo).max() < 1e-13


def test_residual_vs_oracle(solver, oracle):
    N = 64
    pr = P.helmholtz(N, 4.0, seed=11)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = _rand(N, 5)
    r, rel = solver.residual(pr["b"], x)
    gh = oracle.spectrum(pr["g_block"], solver.L)
    ro = oracle.matvec(gh, pr["chi"] * pr["chi_scale"], x, b=pr["b"])
    assert np.abs(r - ro).max() / np.abs(ro).max() < 1e-13
    assert abs(rel - np.linalg.norm(ro) / np.linalg.norm(pr["b"])) < 1e-12 * rel


def test_torch_device_tensors(solver, oracle):
    import torch
    N = 64
    pr = P.helmholtz(N, 2.25, seed=12)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = _rand(N, 6)
    xt = torch.from_numpy(x).cuda()
    yt = solver.matvec(xt)
    assert yt.is_cuda
    y = solver.matvec(x)
    assert np.abs(yt.cpu().numpy() - y).max() == 0.0
