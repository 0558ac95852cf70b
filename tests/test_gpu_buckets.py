"""Lockstep buckets (cugmres_solve_buckets): systems of one grid side solved
together, every Arnoldi-step kernel one launch for the whole bucket.  Each
system must come out as if it had been solved alone: same iteration count
(within one step: the bucket's dot pass reduces over a different number of
blocks, so the sums round differently) and the same solution, checked against
single-system solves and against the oracle's GMRES(m)."""
import numpy as np
import pytest

import cugmres_b200 as cg
from cugmres_b200 import problems as P

pytestmark = pytest.mark.gpu


def _systems():
    rng = np.random.default_rng(7)
    out = []
    for i, N in enumerate((48, 64, 48, 96, 64, 48, 96, 64)):
        out.append(P.helmholtz(N, float(rng.uniform(2.0, 4.0)), seed=100 + i,
                               cells_per_wavelength=float(rng.uniform(15, 30)), with_green=False))
    # a trivial system (eps_r = 1: A = I, one step) and a budget-limited one share buckets with the rest
    out.append(P.helmholtz(64, 1.0, seed=5, with_green=False))
    out.append(P.helmholtz(48, 12.0, seed=6, with_green=False))
    return out


@pytest.mark.parametrize("max_bucket", [0, 2])
def test_buckets_match_single_solves(cuda_device, max_bucket):
    systems = _systems()
    kw = dict(restart=30, max_iter=300, tol=1e-10)
    xs, infos = cg.solve_batch(systems, device=cuda_device, mode="buckets", max_bucket=max_bucket, **kw)
    for sysd, x, info in zip(systems, xs, infos):
        with cg.Solver(cuda_device) as s:
            s.set_operator_green(sysd["N"], sysd["chi"], sysd["chi_scale"], sysd["k0"], sysd["h"])
            xr, ir = s.solve(sysd["b"], **kw)
            _, rel = s.residual(sysd["b"], x)
        assert info["status"] == ir["status"], (sysd["N"], info, ir)
        assert abs(info["iterations"] - ir["iterations"]) <= 1
        assert info["cycles"] == ir["cycles"] or abs(info["iterations"] - ir["iterations"]) == 1
        assert abs(rel - info["rel_residual_true"]) <= 1e-6 * max(rel, 1e-12)
        if ir["status"] == 0:
            assert rel <= 1e-10
            assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-8
        else:
            assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-6
    assert infos[8]["status"] == 0 and infos[8]["iterations"] == 1  # A = I
    assert infos[9]["status"] == cg._lib.CG_ERR_NOT_CONVERGED and infos[9]["iterations"] == 300


def test_bucket_system_matches_oracle(cuda_device, oracle):
    systems = _systems()[:4]
    xs, infos = cg.solve_batch(systems, device=cuda_device, mode="buckets", restart=30, max_iter=400, tol=1e-10)
    sysd, x, info = systems[3], xs[3], infos[3]  # the 96 x 96 system
    g = oracle.green_block_helmholtz(sysd["N"], sysd["k0"], sysd["h"])
    L = 16
    while L < 2 * sysd["N"] - 1:
        L *= 2
    o = oracle.gmres(oracle.spectrum(g, L), sysd["chi"] * sysd["chi_scale"], sysd["b"], restart=30, maxiter=400,
                     tol=1e-10)
    assert info["status"] == 0 and o["status"] == 0
    assert abs(info["iterations"] - o["iterations"]) <= 1
    assert np.linalg.norm(x - o["x"]) / np.linalg.norm(o["x"]) < 1e-9


def test_buckets_mixed_precision_match_single_solves(cuda_device):
    """complex64 cycles with the FP64 residual and update, in lockstep: each
    system converges like its single mixed-precision solve (within two steps:
    the complex64 reductions round differently in a bucket) to the same
    solution, and to 1e-10 in FP64."""
    systems = [s for s in _systems()[:8]]
    kw = dict(restart=30, max_iter=600, tol=1e-10, precision="mixed", inner_tol=1e-5)
    xs, infos = cg.solve_batch(systems, device=cuda_device, mode="buckets", **kw)
    for sysd, x, info in zip(systems, xs, infos):
        with cg.Solver(cuda_device) as s:
            s.set_operator_green(sysd["N"], sysd["chi"], sysd["chi_scale"], sysd["k0"], sysd["h"])
            xr, ir = s.solve(sysd["b"], **kw)
            _, rel = s.residual(sysd["b"], x)
        assert info["status"] == ir["status"], (sysd["N"], info, ir)
        if ir["status"] == 0:
            assert abs(info["iterations"] - ir["iterations"]) <= 2
            assert rel <= 1e-10
            assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-8


def test_buckets_reject_what_they_do_not_run(cuda_device):
    systems = _systems()[:2]
    with pytest.raises(cg.CugmresError):
        cg.solve_batch(systems, device=cuda_device, mode="buckets", ortho="cgs2")
