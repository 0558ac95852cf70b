"""Parity on the benchmark's own system: the 1024 x 1024 GFIEM operator
(eps_r = 4, seed 0, lambda/h = 20; 2048^2 embedding) and the 2048 x 2048 one
(4096^2 embedding), through the C-ABI against the CPU oracle.

The benchmark times exactly these kernel instantiations (FP64 passes at
L = 2048), so they are checked here at that size rather than inferred from
smaller grids."""
import numpy as np
import pytest

from oracle import problems as OP

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system1024(oracle):
    pr = OP.helmholtz(1024, 4.0, seed=0)
    gh = oracle.spectrum(pr["g_block"], OP.embedding(1024))
    return pr, gh


@pytest.mark.parametrize("transpose", [False, True])
def test_matvec_1024_fp64_vs_oracle(solver, oracle, system1024, transpose):
    pr, gh = system1024
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    assert solver.L == 2048
    x = np.random.default_rng(5).standard_normal((1024, 1024)) + 1j * np.random.default_rng(6).standard_normal(
        (1024, 1024))
    c = pr["chi"] * pr["chi_scale"]
    if transpose:
        y, yo = solver.matvec(x, transpose=True), oracle.matvec_transpose(gh, c, x)
    else:
        y, yo = solver.matvec(x), oracle.matvec(gh, c, x)
    assert np.abs(y - yo).max() / np.abs(yo).max() < 1e-13
    y32 = solver.matvec(x.astype(np.complex64), precision="fp32", transpose=transpose)
    assert np.abs(y32 - yo).max() / np.abs(yo).max() < 2e-6


def test_residual_1024_fp64_vs_oracle(solver, oracle, system1024):
    pr, gh = system1024
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = np.random.default_rng(8).standard_normal((1024, 1024)) + 0.5j
    r, rel = solver.residual(pr["b"], x)
    ro = oracle.matvec(gh, pr["chi"] * pr["chi_scale"], x, b=pr["b"])
    assert np.abs(r - ro).max() / np.abs(ro).max() < 1e-13
    assert abs(rel - np.linalg.norm(ro) / np.linalg.norm(pr["b"])) < 1e-12 * rel


def test_matvec_2048_fp64_vs_oracle(solver, oracle):
    N = 2048
    pr = OP.helmholtz(N, 12.25, seed=0)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    assert solver.L == 4096
    gh = oracle.spectrum(pr["g_block"], solver.L)
    x = np.random.default_rng(9).standard_normal((N, N)) - 0.25j
    y = solver.matvec(x)
    yo = oracle.matvec(gh, pr["chi"] * pr["chi_scale"], x)
    assert np.abs(y - yo).max() / np.abs(yo).max() < 1e-13
    y32 = solver.matvec(x.astype(np.complex64), precision="fp32")
    assert np.abs(y32 - yo).max() / np.abs(yo).max() < 2e-6


@pytest.mark.parametrize("ortho", ["dcgs2", "cgs2"])
def test_restart_cycle_1024_fp64_vs_oracle(solver, oracle, system1024, ortho):
    """GMRES(100) on the benchmark system for 110 Arnoldi steps (one whole
    restart cycle, the FP64 residual and update between cycles, and ten steps of
    the next): the GPU iterate matches the oracle's modified Gram-Schmidt GMRES
    (MKL_GMRES.h:225-271 restated) to 1e-10, and the residual history step by
    step.  (The oracle's MGS and CGS2 agree to 2e-13 here.)"""
    pr, gh = system1024
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x, info = solver.solve(pr["b"], restart=100, max_iter=110, tol=0.0, ortho=ortho)
    o = oracle.gmres(gh, pr["chi"] * pr["chi_scale"], pr["b"], restart=100, maxiter=110, tol=0.0)
    assert info["iterations"] == o["iterations"] == 110
    assert info["cycles"] == o["cycles"]
    assert np.linalg.norm(x - o["x"]) / np.linalg.norm(o["x"]) < 1e-10
    assert np.allclose(info["res_hist"][1:], o["res_hist"][1:], rtol=1e-9)
    assert abs(info["rel_residual_true"] - o["true_res"]) < 1e-9 * o["true_res"]


def test_restart_cycle_2048_fp64_vs_oracle(solver, oracle):
    """The config-3 grid (2048^2, 4096^2 embedding, eps_r = 12.25): a GMRES(50)
    run of 55 FP64 Arnoldi steps (one cycle, the residual and update, five
    steps of the next) against the oracle's modified Gram-Schmidt GMRES."""
    N = 2048
    pr = OP.helmholtz(N, 12.25, seed=0)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    assert solver.L == 4096
    gh = oracle.spectrum(pr["g_block"], solver.L)
    x, info = solver.solve(pr["b"], restart=50, max_iter=55, tol=0.0)
    o = oracle.gmres(gh, pr["chi"] * pr["chi_scale"], pr["b"], restart=50, maxiter=55, tol=0.0)
    assert info["iterations"] == o["iterations"] == 55 and info["cycles"] == o["cycles"] == 2
    assert np.linalg.norm(x - o["x"]) / np.linalg.norm(o["x"]) < 1e-10
    assert np.allclose(info["res_hist"][1:], o["res_hist"][1:], rtol=1e-9)
