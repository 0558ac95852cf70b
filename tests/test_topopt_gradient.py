"""The adjoint gradient of the topology-optimisation objective (host logic of
cugmres_b200/topopt.py) against central finite differences, with dense solves
of the operator the oracle's FFT matvec defines (10 x 10 grid, CPU)."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import oracle as O  # noqa: E402
from oracle import problems as OP  # noqa: E402
from cugmres_b200 import topopt  # noqa: E402


def _dense(gh, c, n, N):
    cols = []
    for j in range(n):
        e = np.zeros(n, np.complex128)
        e[j] = 1.0
        cols.append(O.matvec(gh, c, e.reshape(N, N)).reshape(-1))
    return np.stack(cols, axis=1)


def test_adjoint_gradient_matches_finite_differences():
    N = 10
    pr = OP.helmholtz(N, 4.0, seed=2)
    s = pr["chi_scale"]
    gh = O.spectrum(pr["g_block"], OP.embedding(N))
    n = N * N
    b = pr["b"].reshape(-1)
    design = np.zeros((N, N), bool)
    design[3:7, 3:7] = True
    rng = np.random.default_rng(0)
    x = (rng.random((N, N)) > 0.5).astype(np.float64)
    chi_on = 3.0
    chi = np.where(design, chi_on * x, pr["chi"])
    targets = [(8, 5), (1, 2)]
    K = np.eye(n) - _dense(gh, np.ones((N, N)), n, N)

    def solve_state(ch):
        A = _dense(gh, ch * s, n, N)
        return A, np.linalg.solve(A, b).reshape(N, N)

    A, E = solve_state(chi)
    g = topopt.gradient(E, targets, lambda p: np.linalg.solve(A.T, p.reshape(-1)).reshape(N, N),
                        lambda v: (K @ v.reshape(-1)).reshape(N, N), s)
    delta = 1e-6
    for cell in [(4, 4), (2, 7), (6, 3), (8, 5)]:
        cp, cm = chi.copy(), chi.copy()
        cp[cell] += delta
        cm[cell] -= delta
        fd = (topopt.objective(solve_state(cp)[1], targets) - topopt.objective(solve_state(cm)[1], targets)) / (2 * delta)
        assert abs(g[cell] - fd) <= 1e-6 * max(1.0, abs(fd)), (cell, g[cell], fd)


def test_flip_gains_sign_and_mask():
    x = np.array([[0.0, 1.0], [1.0, 0.0]])
    g = np.array([[2.0, 2.0], [-1.0, -1.0]])
    design = np.array([[True, True], [True, False]])
    gain = topopt.flip_gains(x, g, design, 3.0)
    assert gain[0, 0] == 6.0 and gain[0, 1] == -6.0 and gain[1, 0] == 3.0 and gain[1, 1] == -np.inf
