"""Transposed operator A^T x = x - diag(c) G x (the reference's gradient-path
operator and PyGMRES matvec(..., transpose=True)) and the transposed solve."""
import numpy as np
import pytest

from conftest import golden
import cugmres_b200 as cg
from cugmres_b200 import problems as P

pytestmark = pytest.mark.gpu


def _rand(N, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))


@pytest.mark.parametrize("N", [5, 16, 33, 64, 100, 256, 512])
def test_transpose_fp64_vs_oracle(solver, oracle, N):
    pr = P.helmholtz(N, 4.0, seed=N + 1)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = _rand(N, 9)
    y = solver.matvec(x, transpose=True)
    gh = oracle.spectrum(pr["g_block"], solver.L)
    yo = oracle.matvec_transpose(gh, pr["chi"] * pr["chi_scale"], x)
    assert np.abs(y - yo).max() / np.abs(yo).max() < 1e-13


def test_transpose_fp32_vs_oracle(solver, oracle):
    N = 256
    pr = P.helmholtz(N, 4.0, seed=2)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = _rand(N, 4).astype(np.complex64)
    y = solver.matvec(x, precision="fp32", transpose=True)
    gh = oracle.spectrum(pr["g_block"], solver.L)
    yo = oracle.matvec_transpose(gh, pr["chi"] * pr["chi_scale"], x.astype(np.complex128))
    assert np.abs(y - yo).max() / np.abs(yo).max() < 2e-6


@pytest.mark.parametrize("N", [8, 16, 32])
def test_pygmres_transpose_golden(cuda_device, N):
    """cugmres_b200.matvec(..., transpose=True) against the reference's own output."""
    d = golden("pygmres_matvec.npz")
    y = cg.matvec(d[f"x_{N}"], d[f"eps_{N}"], float(d[f"k_{N}"]), transpose=True)
    yt = d[f"yt_{N}"]
    assert np.abs(y.ravel() - yt).max() / np.abs(yt).max() < 2e-7


def test_transpose_is_the_transpose(solver):
    """<A^T x, y> = <x, A y> (bilinear, no conjugation)."""
    N = 64
    pr = P.helmholtz(N, 6.0, seed=3)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x, y = _rand(N, 1), _rand(N, 2)
    lhs = np.sum(solver.matvec(x, transpose=True) * y)
    rhs = np.sum(x * solver.matvec(y))
    assert abs(lhs - rhs) <= 1e-12 * abs(rhs)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_transposed_solve(solver, oracle, precision):
    """Solve A^T x = e_i (the reference's gradient right-hand side, a unit vector)."""
    N = 64
    pr = P.helmholtz(N, 4.0, seed=5)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    b = np.zeros((N, N), np.complex128)
    b[N // 2, N // 3] = 1.0
    x, info = solver.solve(b, restart=200, max_iter=3000, tol=1e-10, precision=precision, transpose=True)
    assert info["status"] == 0
    gh = oracle.spectrum(pr["g_block"], solver.L)
    r = b - oracle.matvec_transpose(gh, pr["chi"] * pr["chi_scale"], x)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.01e-10
    assert abs(info["rel_residual_true"] - np.linalg.norm(r) / np.linalg.norm(b)) < 1e-12
