"""Batched sweep (cugmres_solve_batch): concurrent contexts give the same
per-system results as one solve at a time."""
import numpy as np
import pytest

import cugmres_b200 as cg
from cugmres_b200 import problems as P

pytestmark = pytest.mark.gpu


def test_batch_matches_single_solves(cuda_device):
    systems = P.sweep(nsys=12, seed=3, sides=(16, 24, 40, 64, 100), lam_over_h=(15, 30), eps_range=(1.5, 3.0))
    xs, infos = cg.solve_batch(systems, device=cuda_device, workers=4, restart=60, max_iter=3000, tol=1e-10)
    for s, x, info in zip(systems, xs, infos):
        with cg.Solver(cuda_device) as solver:
            solver.set_operator(s["g_block"], s["chi"], s["chi_scale"])
            x1, i1 = solver.solve(s["b"], restart=60, max_iter=3000, tol=1e-10)
        assert info["status"] == i1["status"] == 0
        assert info["iterations"] == i1["iterations"]
        assert info["rel_residual_true"] <= 1e-10
        assert np.linalg.norm(x - x1) / np.linalg.norm(x1) < 1e-12
        assert info["seconds"] > 0


def test_batch_reports_per_system_status(cuda_device):
    systems = P.sweep(nsys=4, seed=5, sides=(32, 48), eps_range=(3.0, 4.0))
    xs, infos = cg.solve_batch(systems, device=cuda_device, workers=2, restart=5, max_iter=5, tol=1e-14)
    assert all(i["status"] == cg._lib.CG_ERR_NOT_CONVERGED and i["iterations"] == 5 for i in infos)
