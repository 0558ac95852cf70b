"""GPU GMRES (CGS2 + single-warp Givens, device-side control) against the CPU
oracle's restatement of the reference method, through the C-ABI."""
import numpy as np
import pytest

from conftest import golden
import cugmres_b200 as cg
from cugmres_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,maxit", [(64, 60), (128, 50)])
def test_reference_semantics_vs_oracle(solver, oracle, N, maxit):
    """Fixed maxiter, reference Givens formula, x0 = b: the FP64 solution matches
    the complex128 restatement of FFT_GMRES_with_MKL to 1e-10.

    The reference's rotation is not unitary for complex diagonals, which makes
    unconverged iterates extremely sensitive to rounding: two CPU restatements
    (MGS with explicit Jtotal + LU, and CGS2 with (c, s) pairs) already differ
    by 4e-9 after 20 steps and 3.5e-3 after 30 steps at N=64.  The step counts
    here reach convergence (true residual ~1e-14), where they agree to 1e-14."""
    pr = P.reference_cylinder(N)
    solver.set_operator(pr["g_block"], pr["chi"], 1.0)
    x, info = solver.solve(pr["b"], x0=pr["x0"], restart=maxit, max_iter=maxit, tol=1e-8,
                           givens="reference", fixed_iterations=True)
    gh = oracle.spectrum(pr["g_block"], solver.L)
    xo, res, n, flag, _ = oracle.gmres_reference(gh, pr["chi"], pr["b"], pr["x0"], maxit, 1e-8)
    assert info["iterations"] == n == maxit
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-10
    # Residual estimates: the faithful restatement accumulates Jtotal by explicit
    # products, whose rounding moves mid-run estimates by up to 60 % on these
    # cases even between two CPU restatements; the history is therefore compared
    # with the oracle's (c, s)-pair formulation of the same method.
    o = oracle.gmres(gh, pr["chi"], pr["b"], x0=pr["x0"], restart=maxit, maxiter=maxit, tol=0.0, ortho="cgs2",
                     rotation="reference")
    # first 20 steps only: on these cases the estimates of any two implementations
    # (even the CPU oracle's MGS and CGS2) deviate by more than 1e-6 from step 23
    # on and by up to 40 % later, while the converged solutions agree to 1e-14
    assert np.allclose(info["res_hist"][:21], o["res_hist"][:21], rtol=1e-6)


def test_mkl_solution_256_on_gpu(solver, oracle):
    N = 256
    d = golden("ref_mkl_solution_256_m44.npz")
    ref = d["solution"].astype(np.complex128)
    pr = P.reference_cylinder(N)
    solver.set_operator(pr["g_block"], pr["chi"], 1.0)
    x, info = solver.solve(pr["b"], x0=pr["x0"], restart=44, max_iter=44, tol=1e-8, givens="reference",
                           fixed_iterations=True)
    assert info["iterations"] == 44
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 3e-5
    gh = oracle.spectrum(pr["g_block"], solver.L)
    xo, *_ = oracle.gmres_reference(gh, pr["chi"], pr["b"], pr["x0"], 44, 1e-8)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-10


def test_fast_gmres_drop_in(cuda_device, oracle):
    N, maxit = 64, 60
    gp = golden("ref_G_prep_64.npz")["g_prep"]
    pr = P.reference_cylinder(N)
    sol, res, n, flag = cg.fast_gmres(gp, pr["mask"], pr["x0"].astype(np.complex64), maxit, 1e-3, pr["chi_value"])
    assert n == maxit and res.shape == (maxit + 1,)
    gh = oracle.spectrum(gp[:N, :N].astype(np.complex128), 2 * N)
    xo, reso, no, flago, _ = oracle.gmres_reference(gh, pr["chi"], pr["b"], pr["x0"], maxit, 1e-3)
    assert np.linalg.norm(sol - xo) / np.linalg.norm(xo) < 1e-6  # complex64 output
    assert abs(res[0] - reso[0]) < 1e-5 * reso[0]
    o = oracle.gmres(gh, pr["chi"], pr["b"], x0=pr["x0"], restart=maxit, maxiter=maxit, tol=0.0, ortho="cgs2",
                     rotation="reference")
    est = o["res_hist"] * np.linalg.norm(pr["b"])
    assert np.allclose(res[:21], est[:21], rtol=1e-5)  # see test_reference_semantics_vs_oracle
    assert flag == (res[-1] > 1e-3)


@pytest.mark.parametrize("restart", [10, 30])
def test_restarted_unitary_vs_oracle(solver, oracle, restart):
    """Same number of steps, same restart: GPU CGS2 and oracle MGS iterates agree."""
    N = 48
    pr = P.helmholtz(N, 2.25, seed=21)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x, info = solver.solve(pr["b"], restart=restart, max_iter=60, tol=0.0)
    gh = oracle.spectrum(pr["g_block"], solver.L)
    o = oracle.gmres(gh, pr["chi"] * pr["chi_scale"], pr["b"], restart=restart, maxiter=60, tol=0.0)
    assert info["iterations"] == o["iterations"] == 60
    assert np.linalg.norm(x - o["x"]) / np.linalg.norm(o["x"]) < 1e-10
    assert np.allclose(info["res_hist"][1:], o["res_hist"][1:], rtol=1e-7)


def test_config1_64_converges_like_oracle(solver, oracle):
    """64x64, eps_r = 2.25, unrestarted, tol 1e-10, max 500: iterations within +-1 of
    the oracle, FP64 true residual <= 1e-10, error vs a 1e-13 FP64 solve."""
    N = 64
    pr = P.helmholtz(N, 2.25, seed=0)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x, info = solver.solve(pr["b"], restart=500, max_iter=500, tol=1e-10)
    assert info["status"] == 0
    assert info["rel_residual_true"] <= 1e-10
    gh = oracle.spectrum(pr["g_block"], solver.L)
    c = pr["chi"] * pr["chi_scale"]
    o = oracle.gmres(gh, c, pr["b"], restart=500, maxiter=500, tol=1e-10)
    assert abs(info["iterations"] - o["iterations"]) <= 1
    assert np.linalg.norm(x - o["x"]) / np.linalg.norm(o["x"]) < 1e-9
    tight = oracle.gmres(gh, c, pr["b"], restart=500, maxiter=500, tol=1e-13)
    assert np.linalg.norm(x - tight["x"]) / np.linalg.norm(tight["x"]) < 1e-8


def test_mixed_precision_refinement(solver, oracle):
    N = 128
    pr = P.helmholtz(N, 2.25, seed=2)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x, info = solver.solve(pr["b"], restart=50, max_iter=3000, tol=1e-10, precision="mixed", inner_tol=1e-5)
    assert info["status"] == 0 and info["rel_residual_true"] <= 1e-10
    x64, info64 = solver.solve(pr["b"], restart=50, max_iter=3000, tol=1e-13)
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-8
    _, rel = solver.residual(pr["b"], x)
    assert rel <= 1e-10


def test_identity_operator_happy_breakdown(solver):
    N = 32
    pr = P.helmholtz(N, 1.0, seed=0)  # eps_r = 1 -> chi = 0 -> A = I
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x, info = solver.solve(pr["b"], restart=10, max_iter=10, tol=1e-12)
    assert info["status"] == 0 and info["iterations"] == 1
    assert np.abs(x - pr["b"]).max() < 1e-14


def test_status_codes(solver):
    N = 32
    pr = P.helmholtz(N, 4.0, seed=0)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x, info = solver.solve(pr["b"], restart=5, max_iter=5, tol=1e-14)
    assert info["status"] == cg._lib.CG_ERR_NOT_CONVERGED and info["iterations"] == 5
    bad = pr["b"].copy()
    bad[3, 4] = np.nan
    x, info = solver.solve(bad, restart=5, max_iter=5)
    assert info["status"] == cg._lib.CG_ERR_NONFINITE
    with pytest.raises(cg.CugmresError):
        solver.solve(pr["b"], restart=0)
    x, info = solver.solve(pr["b"], restart=50, max_iter=100000, tol=1e-30, timeout_s=0.2)
    assert info["status"] == cg._lib.CG_ERR_TIMEOUT


def test_device_resident_solve(solver):
    import torch
    N = 64
    pr = P.helmholtz(N, 2.25, seed=7)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    bt = torch.from_numpy(pr["b"]).cuda()
    xt, info = solver.solve(bt, restart=100, max_iter=500, tol=1e-10)
    assert xt.is_cuda and info["status"] == 0
    x, info2 = solver.solve(pr["b"], restart=100, max_iter=500, tol=1e-10)
    assert info["iterations"] == info2["iterations"]
    assert np.abs(xt.cpu().numpy() - x).max() == 0.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_delayed_and_immediate_reorthogonalisation_agree(solver, precision):
    """The delayed CGS2 (2 basis passes per step) and plain CGS2 (4 passes) give
    the same iterates: same iteration count, same residual history."""
    N = 96
    pr = P.helmholtz(N, 2.25, seed=31)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    kw = dict(restart=40, max_iter=2000, tol=1e-10, precision=precision)
    xa, ia = solver.solve(pr["b"], ortho="dcgs2", **kw)
    xb, ib = solver.solve(pr["b"], ortho="cgs2", **kw)
    assert ia["status"] == ib["status"] == 0
    assert abs(ia["iterations"] - ib["iterations"]) <= (0 if precision == "fp64" else 2)
    assert np.linalg.norm(xa - xb) / np.linalg.norm(xb) < (1e-9 if precision == "fp64" else 1e-8)
    n = min(len(ia["res_hist"]), len(ib["res_hist"]), 40)
    live = ib["res_hist"][:n] > 1e-8
    assert np.allclose(ia["res_hist"][:n][live], ib["res_hist"][:n][live], rtol=1e-6 if precision == "fp64" else 1e-3)
