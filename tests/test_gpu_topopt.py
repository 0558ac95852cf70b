"""Topology optimisation on the GPU solver (cugmres_b200/topopt.py): the
adjoint gradient from the transposed solve against finite differences of the
objective, and the discrete-gradient and greedy searches raising the field
intensity at one and at two target points of a 32 x 32 design."""
import numpy as np
import pytest

import cugmres_b200 as cg
from cugmres_b200 import problems as P
from cugmres_b200 import topopt

pytestmark = pytest.mark.gpu

N = 32


def _problem(device):
    pr = P.helmholtz(N, 1.0, seed=0)  # eps_r = 1: free space outside the design
    design = np.zeros((N, N), bool)
    design[8:20, 10:22] = True
    prob = topopt.Problem(pr["g_block"], np.zeros((N, N)), design, chi_on=3.0, s=pr["chi_scale"], b=pr["b"],
                          device=device, restart=200, tol=1e-12)
    return pr, prob


def test_gradient_matches_finite_differences(cuda_device):
    pr, prob = _problem(cuda_device)
    try:
        rng = np.random.default_rng(1)
        x = np.where(prob.design, (rng.random((N, N)) > 0.5).astype(np.float64), 0.0)
        targets = [(26, 16)]
        F, g, _ = prob.value_and_gradient(x, targets)
        chi = prob.chi(x)
        delta = 1e-5
        with cg.Solver(cuda_device) as s:
            def F_of(ch):
                s.set_operator(pr["g_block"], ch, pr["chi_scale"])
                E, info = s.solve(pr["b"], restart=200, tol=1e-13, max_iter=20000)
                assert info["status"] == 0
                return topopt.objective(E, targets)
            for cell in [(12, 14), (18, 20), (26, 16), (3, 3)]:
                cp, cm = chi.copy(), chi.copy()
                cp[cell] += delta
                cm[cell] -= delta
                fd = (F_of(cp) - F_of(cm)) / (2 * delta)
                assert abs(g[cell] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(g).max()), (cell, g[cell], fd)
    finally:
        prob.close()


# two focal points compete for the same design cells: a smaller gain in 8 moves
@pytest.mark.parametrize("targets, gain", [([(26, 16)], 2.0), ([(26, 12), (26, 20)], 1.4)])
def test_discrete_gradient_raises_intensity(cuda_device, targets, gain):
    _, prob = _problem(cuda_device)
    try:
        x, hist = topopt.discrete_gradient(prob, np.zeros((N, N)), targets, iterations=8)
        F = [h[0] for h in hist]
        assert len(F) >= 3 and all(b > a for a, b in zip(F, F[1:])), F
        assert F[-1] > gain * F[0], F
        assert set(np.unique(x)) <= {0.0, 1.0} and not np.any(x[~prob.design])
        assert abs(topopt.objective(prob.forward(x), targets) - F[-1]) <= 1e-9 * F[-1]
    finally:
        prob.close()


def test_greedy_raises_intensity(cuda_device):
    _, prob = _problem(cuda_device)
    try:
        x, hist = topopt.greedy(prob, np.zeros((N, N)), [(26, 16)], iterations=4)
        F = [h[0] for h in hist]
        assert len(F) >= 2 and all(b > a for a, b in zip(F, F[1:])), F
        assert int(np.sum(x)) == len(F) - 1  # one accepted flip per step from the empty design
    finally:
        prob.close()
