"""Topology optimisation of a photonic design on the GFIEM system (the
application the reference's drivers address: discrete-gradient and greedy
searches over binary permittivity designs, with one or several target points;
`CUDA_GMRES/main.cu:20-28` names `discrete_gradient_numerical_method_v1..v3`,
`greedy_numerical_method_v1` and `discrete_gradient_multiple_points_*`, whose
sources the reference does not ship).  Written from the adjoint method:

  state      A(chi) E = b,  A = I - K diag(s chi),  K the BTTB Green's matrix
             (symmetric), s the contrast scale (k0^2);
  objective  F = sum_t |E_t|^2 over the target cells t;
  gradient   dF/dchi_i = 2 s Re(w_i E_i),  w = K y,  A^T y = p,
             p = sum_t conj(E_t) e_t,
             because dA/dchi_i = -s K e_i e_i^T and A K = K A^T.

A^T y = p is the reference's gradient solve (`for_gradient`: the transposed
operator with the contrast moved to the crop, a unit right-hand side at the
target, `CUDA_GMRES/GMRES.cuh:97-111`); w = K y uses a second operator with
unit contrast (K v = v - A_1 v).  The design is binary: chi_i = chi_on x_i on
the design cells (x_i in {0, 1}), fixed elsewhere.

The search moves (flip a cell where the first-order change of F is positive,
largest first; halve the step when the objective does not rise) and the
greedy variant (one flip per forward solve, keep it only if F rises) are this
module's own, built on those gradients.  Every solve is the GPU GMRES of this
library; the per-cell arithmetic is NumPy on N^2 values.
"""
import numpy as np


def objective(E, targets):
    """F = sum over target cells (row, col) of |E|^2."""
    return float(sum(abs(E[r, c]) ** 2 for r, c in targets))


def gradient(E, targets, solve_adjoint, apply_k, s):
    """dF/dchi for every cell: 2 s Re(w E), w = K y, A^T y = p.
    solve_adjoint(p) returns y with A^T y = p; apply_k(v) returns K v."""
    p = np.zeros_like(E)
    for r, c in targets:
        p[r, c] += np.conj(E[r, c])
    y = solve_adjoint(p)
    w = apply_k(y)
    return 2.0 * s * np.real(w * E)


class Problem:
    """Forward and adjoint solves of one design on one GPU.

    g_block: the N x N Green's block; chi_fixed: the contrast outside the
    design (N x N); design: boolean mask of the design cells; chi_on: the
    contrast of a filled design cell; s: contrast scale (k0^2); b: incident
    field.  Solves run to `tol` with GMRES(`restart`)."""

    def __init__(self, g_block, chi_fixed, design, chi_on, s, b, device=0, restart=200, tol=1e-11,
                 max_iter=20000, precision="fp64"):
        import cugmres_b200 as cg
        self.N = g_block.shape[0]
        self.g_block = np.asarray(g_block)
        self.chi_fixed = np.asarray(chi_fixed, np.float64)
        self.design = np.asarray(design, bool)
        self.chi_on = float(chi_on)
        self.s = float(s)
        self.b = np.asarray(b, np.complex128)
        self.kw = dict(restart=restart, tol=tol, max_iter=max_iter, precision=precision)
        self.solver = cg.Solver(device)
        self.kop = cg.Solver(device)  # unit contrast: K v = v - A_1 v
        self.kop.set_operator(self.g_block, np.ones((self.N, self.N)), 1.0)
        self.solves = 0
        self._x = None

    def close(self):
        self.solver.close()
        self.kop.close()

    def chi(self, x):
        return np.where(self.design, self.chi_on * x, self.chi_fixed)

    def set_design(self, x):
        x = np.asarray(x, np.float64)
        if self._x is None or not np.array_equal(x, self._x):
            self.solver.set_operator(self.g_block, self.chi(x), self.s)
            self._x = x.copy()

    def forward(self, x):
        self.set_design(x)
        E, info = self.solver.solve(self.b, **self.kw)
        self.solves += 1
        if info["status"] != 0:
            raise RuntimeError(f"forward solve: {info['status_text']}")
        return E

    def adjoint(self, x, p):
        self.set_design(x)
        y, info = self.solver.solve(p, transpose=True, **self.kw)
        self.solves += 1
        if info["status"] != 0:
            raise RuntimeError(f"adjoint solve: {info['status_text']}")
        return y

    def apply_k(self, v):
        return v - self.kop.matvec(v)

    def value_and_gradient(self, x, targets):
        E = self.forward(x)
        g = gradient(E, targets, lambda p: self.adjoint(x, p), self.apply_k, self.s)
        return objective(E, targets), g, E


def flip_gains(x, g, design, chi_on):
    """First-order change of F when cell i flips: g_i * chi_on * (1 - 2 x_i)
    on design cells, -inf elsewhere."""
    gain = g * chi_on * (1.0 - 2.0 * x)
    return np.where(design, gain, -np.inf)


def discrete_gradient(prob, x0, targets, iterations=20, step=None, min_step=1):
    """Discrete-gradient search: flip the `step` design cells with the
    largest positive first-order gains; keep the move if F rises (then grow
    the step by half), otherwise halve the step and retry from the same
    design.  Returns (x, history of (F, step, flips))."""
    x = np.asarray(x0, np.float64).copy()
    ncell = int(prob.design.sum())
    step = step or max(1, ncell // 20)
    F, g, _ = prob.value_and_gradient(x, targets)
    hist = [(F, 0, 0)]
    for _ in range(iterations):
        gain = flip_gains(x, g, prob.design, prob.chi_on)
        order = np.argsort(gain, axis=None)[::-1]
        pos = int(np.sum(gain > 0))
        if pos == 0:
            break
        while step >= min_step:
            take = order[:min(step, pos)]
            xt = x.copy()
            xt.flat[take] = 1.0 - xt.flat[take]
            Ft, gt, _ = prob.value_and_gradient(xt, targets)
            if Ft > F:
                x, F, g = xt, Ft, gt
                hist.append((F, step, len(take)))
                step = max(step + step // 2, step + 1)
                break
            step //= 2
        else:
            break
    return x, hist


def greedy(prob, x0, targets, iterations=20, candidates=8):
    """Greedy search: per iteration, try the `candidates` cells with the
    largest first-order gains one at a time (one forward solve each) and
    keep the first flip that raises F; gradients are refreshed after each
    accepted flip.  Returns (x, history of (F, cell))."""
    x = np.asarray(x0, np.float64).copy()
    F, g, _ = prob.value_and_gradient(x, targets)
    hist = [(F, -1)]
    for _ in range(iterations):
        gain = flip_gains(x, g, prob.design, prob.chi_on)
        order = np.argsort(gain, axis=None)[::-1][:candidates]
        moved = False
        for cell in order:
            if not gain.flat[cell] > 0:
                break
            xt = x.copy()
            xt.flat[cell] = 1.0 - xt.flat[cell]
            Ft = objective(prob.forward(xt), targets)
            if Ft > F:
                x, F = xt, Ft
                hist.append((F, int(cell)))
                F, g, _ = prob.value_and_gradient(x, targets)
                moved = True
                break
        if not moved:
            break
    return x, hist
