"""cugmres_b200 -- B200-native GMRES for A = I - G diag(c) on an N x N grid.

G is the symmetric block-Toeplitz-Toeplitz-block Green's-function matrix of
the 2D Helmholtz Lippmann-Schwinger (GFIEM) equation and c = k0^2 chi the
scaled contrast.  The solver is hand-written sm_100a CUDA behind the C-ABI in
include/cugmres.h (libcugmres.so); this module is the Python front-end:

* ``Solver`` -- a context with an operator, ``matvec``, ``residual``, ``solve``.
* PyGMRES-compatible helpers with the signatures of the reference's NumPy
  module (PyGMRES/GMRES.py:13-69): ``get_plane_wave``, ``get_green_matrix``, ``get_toeplitz_mat``, ``get_eps_from_mask``,
  ``matvec`` -- the operator application runs on the GPU.
* ``fast_gmres`` -- the reference's Fast_GMRES_with_CUDA semantics
  (CUDA_GMRES/GMRES.cuh:22-35) in complex64.

Inputs may be NumPy arrays (host) or contiguous torch tensors (host or CUDA);
the C library detects device pointers itself.  There is no CPU fallback: a
missing library or a failing CUDA call raises.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import CugmresError, check
from .problems import green_block, helmholtz, reference_cylinder

__all__ = ["Solver", "CugmresError", "green_block", "helmholtz", "reference_cylinder", "matvec", "solve_batch",
           "get_plane_wave", "get_green_matrix", "get_toeplitz_mat", "get_eps_from_mask",
           "fast_gmres", "gmres"]

_PREC = {"fp64": _lib.CG_PREC_FP64, "mixed": _lib.CG_PREC_MIXED, "fp32": _lib.CG_PREC_MIXED}
_GIV = {"unitary": _lib.CG_GIVENS_UNITARY, "reference": _lib.CG_GIVENS_REFERENCE}
_ORTHO = {"dcgs2": _lib.CG_ORTHO_DCGS2, "cgs2": _lib.CG_ORTHO_CGS2, "sstep": _lib.CG_ORTHO_SSTEP}


def _is_torch(a):
    return type(a).__module__.split(".")[0] == "torch"


def _np_dtype_name(dt):
    return {np.complex128: "complex128", np.complex64: "complex64", np.float64: "float64",
            np.float32: "float32", np.uint8: "uint8"}[dt]


def _arg(a, dtype, copy=False):
    """(c_void_p, keepalive) for a NumPy array or a contiguous torch tensor."""
    if _is_torch(a):
        name = _np_dtype_name(dtype)
        if str(a.dtype) != "torch." + name:
            raise TypeError(f"expected torch.{name}, got {a.dtype}")
        if not a.is_contiguous():
            raise TypeError("tensor must be contiguous")
        return ctypes.c_void_p(a.data_ptr()), a
    arr = np.array(a, dtype=dtype, order="C", copy=True) if copy else np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data_as(ctypes.c_void_p), arr


class Solver:
    """One solver context (device workspace + CUDA stream) on ``device``."""

    def __init__(self, device=0):
        self._ctx = ctypes.c_void_p()
        check(_lib.lib().cugmres_create(ctypes.byref(self._ctx), int(device)), "cugmres_create")
        self.N = None
        self.L = None

    def close(self):
        if self._ctx:
            _lib.lib().cugmres_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _grid(self):
        N, L = ctypes.c_int(0), ctypes.c_int(0)
        check(_lib.lib().cugmres_grid_size(self._ctx, ctypes.byref(N), ctypes.byref(L)), "grid_size")
        self.N, self.L = N.value, L.value

    def set_stream(self, stream):
        """Run on a caller's cudaStream_t (an int handle, e.g. torch's stream.cuda_stream)."""
        check(_lib.lib().cugmres_set_stream(self._ctx, ctypes.c_void_p(int(stream))), "set_stream")

    def synchronize(self):
        check(_lib.lib().cugmres_synchronize(self._ctx), "synchronize")

    def matvec_shapes(self, precision="fp64"):
        """Autotuned launch shapes (row forward, column convolution, row inverse)."""
        arr = (ctypes.c_int * 3)()
        check(_lib.lib().cugmres_matvec_shapes(self._ctx, _PREC[precision], arr), "matvec_shapes")
        return tuple(arr)

    def profile(self, enable=True):
        """Enable (and reset) per-phase device timing of solve()."""
        check(_lib.lib().cugmres_profile(self._ctx, int(bool(enable))), "profile")

    def profile_read(self):
        """{phase: dict(ms, bytes, launches, gbs)} accumulated since profile(True)."""
        arr = (_lib.CgPhaseStats * len(_lib.PHASES))()
        check(_lib.lib().cugmres_profile_read(self._ctx, arr), "profile_read")
        out = {}
        for name, st in zip(_lib.PHASES, arr):
            out[name] = dict(ms=st.ms, bytes=st.bytes, launches=st.launches,
                             gbs=(st.bytes / (st.ms * 1e-3) / 1e9) if st.ms > 0 else 0.0)
        return out

    def set_operator(self, g_block, chi, chi_scale=1.0):
        """A = I - G diag(chi_scale * chi); g_block[d1, d2] is G at offset (d1, d2)."""
        N = int(g_block.shape[0])
        gp, gk = _arg(g_block, np.complex128)
        cp, ck = _arg(chi, np.float64)
        check(_lib.lib().cugmres_set_operator(self._ctx, N, gp, cp, float(chi_scale)), "set_operator")
        self._grid()
        return self

    def set_operator_circulant(self, g_prep, chi, chi_scale=1.0):
        """Operator from the reference's spatial (2N-1)^2 circulant (G_prep layout)."""
        M = int(g_prep.shape[0])
        N = (M + 1) // 2
        gp, gk = _arg(g_prep, np.complex64)
        cp, ck = _arg(chi, np.float64)
        check(_lib.lib().cugmres_set_operator_circulant(self._ctx, N, gp, cp, float(chi_scale)),
              "set_operator_circulant")
        self._grid()
        return self

    def set_operator_green(self, N, chi, chi_scale, k0=0.0, h=0.0, kind="helmholtz"):
        """Operator set-up entirely on the GPU: Green's block of `kind` ('helmholtz',
        'reference', 'pygmres'), embedding and spectrum; only chi is copied."""
        kinds = {"helmholtz": _lib.CG_GREEN_HELMHOLTZ, "reference": _lib.CG_GREEN_REFERENCE,
                 "pygmres": _lib.CG_GREEN_PYGMRES}
        cp, ck = _arg(chi, np.float64)
        check(_lib.lib().cugmres_set_operator_green(self._ctx, kinds[kind], int(N), float(k0), float(h), cp,
                                                    float(chi_scale)), "set_operator_green")
        self._grid()
        return self

    def matvec(self, x, precision="fp64", out=None, transpose=False):
        """y = A x (transpose: y = A^T x = x - diag(c) G x); precision 'fp64'
        (complex128) or 'fp32' (complex64)."""
        prec = _PREC[precision]
        dt = np.complex128 if prec == _lib.CG_PREC_FP64 else np.complex64
        xp, xk = _arg(x, dt)
        if out is None:
            out = np.empty((self.N, self.N), dt) if not _is_torch(x) else x.new_empty(x.shape)
        yp, yk = _arg(out, dt)
        fn = _lib.lib().cugmres_matvec_transpose if transpose else _lib.lib().cugmres_matvec
        check(fn(self._ctx, xp, yp, prec), "matvec")
        return yk

    def residual(self, b, x):
        """(r, ||r|| / ||b||) with r = b - A x in FP64."""
        bp, bk = _arg(b, np.complex128)
        xp, xk = _arg(x, np.complex128)
        r = np.empty((self.N, self.N), np.complex128)
        rel = ctypes.c_double(0.0)
        check(_lib.lib().cugmres_residual(self._ctx, bp, xp, r.ctypes.data_as(ctypes.c_void_p),
                                          ctypes.byref(rel)), "residual")
        return r, rel.value

    def set_preconditioner(self, net, k0h=None):
        """Attach a learned.FNO (or None to detach) for solve(preconditioner="learned");
        k0h = k0 * h of the current operator."""
        if net is None:
            check(_lib.lib().cugmres_set_preconditioner(self._ctx, None, 0.0), "set_preconditioner")
            self._net = None
            return
        check(_lib.lib().cugmres_set_preconditioner(self._ctx, net._net, float(k0h)), "set_preconditioner")
        self._net = net  # keep the network alive while attached

    def solve(self, b, x0=None, restart=100, max_iter=10000, tol=1e-10, precision="fp64", givens="unitary",
              inner_tol=1e-5, fixed_iterations=False, timeout_s=0.0, ortho="dcgs2", raise_on_failure=False,
              preconditioner=None, learned_x0=False, transpose=False, sstep=4):
        """Solve A x = b.  Returns (x, info) where info holds status, iterations,
        cycles, rel_residual_true / _estimate, seconds and res_hist.
        preconditioner="learned": flexible GMRES with the attached network
        (learned_x0: also start from x0 = M(b) when x0 is None).
        transpose=True solves A^T x = b (the adjoint system of the gradient path).
        ortho="sstep": s-step Arnoldi, `sstep` (2, 4 or 8) steps per block; the
        Newton shifts come from a 24-step delayed-CGS2 run made before the solve."""
        o = _lib.CgOpts()
        _lib.lib().cugmres_default_opts(ctypes.byref(o))
        o.restart = int(restart)
        o.max_iter = int(max_iter)
        o.tol = float(tol)
        o.precision = _PREC[precision]
        o.givens = _GIV[givens]
        o.inner_tol = float(inner_tol)
        o.fixed_iterations = int(bool(fixed_iterations))
        o.timeout_s = float(timeout_s)
        o.ortho = _ORTHO[ortho]
        o.sstep = int(sstep)
        o.preconditioner = {None: 0, "none": 0, "learned": 1}[preconditioner]
        o.learned_x0 = int(bool(learned_x0))
        o.transpose = int(bool(transpose))
        bp, bk = _arg(b, np.complex128)
        if x0 is None:
            o.zero_x0 = 1
            x = np.zeros((self.N, self.N), np.complex128) if not _is_torch(b) else b.new_zeros(b.shape)
        else:
            x = x0 if _is_torch(x0) else np.array(x0, dtype=np.complex128, order="C", copy=True)
        xp, xk = _arg(x, np.complex128)
        hist = np.zeros(int(max_iter) + 1, np.float64)
        res = _lib.CgResult()
        st = _lib.lib().cugmres_solve(self._ctx, bp, xp, ctypes.byref(o), hist.ctypes.data_as(ctypes.c_void_p),
                                      len(hist), ctypes.byref(res))
        if st in (_lib.CG_ERR_INVALID, _lib.CG_ERR_CUDA, _lib.CG_ERR_OOM, _lib.CG_ERR_NO_OPERATOR,
                  _lib.CG_ERR_NOT_IMPLEMENTED) or (raise_on_failure and st != _lib.CG_OK):
            raise CugmresError(st, "cugmres_solve")
        info = dict(status=st, status_text=_lib.strerror(st), iterations=res.iterations, cycles=res.cycles,
                    rel_residual_estimate=res.rel_residual_estimate, rel_residual_true=res.rel_residual_true,
                    seconds=res.seconds, res_hist=hist[: res.iterations + 1].copy(),
                    preconditioned_cycles=res.preconditioned_cycles, x0_learned=res.x0_learned)
        return xk, info


def solve_batch(systems, device=0, workers=8, restart=100, max_iter=10000, tol=1e-10, precision="fp64",
                givens="unitary", inner_tol=1e-5, ortho="dcgs2", device_green=False, mode="buckets", max_bucket=0):
    """Solve many independent systems.

    mode="buckets" (cugmres_solve_buckets): systems of one grid side are solved
    in lockstep, every Arnoldi-step kernel one launch for the whole bucket and
    every restart cycle one CUDA-graph replay (FP64, delayed CGS2; max_bucket
    caps the systems per bucket, 0 = as many as fit in half the free memory).
    mode="contexts" (cugmres_solve_batch): `workers` concurrent contexts, each
    with its own stream, take systems largest first (any precision / scheme).

    systems: iterable of dicts with g_block (or k0 and h: the GFIEM block is
    then built on the GPU; device_green=True forces that), chi, chi_scale, b
    and optionally x0.
    Returns (xs, infos): solutions (complex128 N x N) and per-system dicts with
    status, iterations, rel_residual_true and seconds (latency)."""
    systems = list(systems)
    keep, arr = [], (_lib.CgSystem * max(1, len(systems)))()
    xs = []
    for i, sysd in enumerate(systems):
        c = np.ascontiguousarray(sysd["chi"], np.float64)
        N = int(c.shape[0])
        g = None if device_green or sysd.get("g_block") is None else np.ascontiguousarray(sysd["g_block"], np.complex128)
        b = np.ascontiguousarray(sysd["b"], np.complex128)
        x = np.zeros((N, N), np.complex128) if sysd.get("x0") is None else np.array(sysd["x0"], np.complex128)
        keep += [g, c, b]
        xs.append(x)
        arr[i] = _lib.CgSystem(N, g.ctypes.data if g is not None else None, c.ctypes.data,
                               float(sysd.get("chi_scale", 1.0)), b.ctypes.data, x.ctypes.data,
                               float(sysd.get("k0", 0.0)), float(sysd.get("h", 0.0)))
    o = _lib.CgOpts()
    _lib.lib().cugmres_default_opts(ctypes.byref(o))
    o.restart, o.max_iter, o.tol = int(restart), int(max_iter), float(tol)
    o.precision, o.givens, o.inner_tol, o.ortho = _PREC[precision], _GIV[givens], float(inner_tol), _ORTHO[ortho]
    res = (_lib.CgResult * max(1, len(systems)))()
    if mode == "buckets":
        o.zero_x0 = int(all(sysd.get("x0") is None for sysd in systems))
        check(_lib.lib().cugmres_solve_buckets(int(device), len(systems), arr, ctypes.byref(o), int(max_bucket), res),
              "cugmres_solve_buckets")
    elif mode == "contexts":
        check(_lib.lib().cugmres_solve_batch(int(device), len(systems), arr, ctypes.byref(o), int(workers), res),
              "cugmres_solve_batch")
    else:
        raise ValueError(mode)
    infos = [dict(status=r.status, status_text=_lib.strerror(r.status), iterations=r.iterations, cycles=r.cycles,
                  rel_residual_true=r.rel_residual_true, rel_residual_estimate=r.rel_residual_estimate,
                  seconds=r.seconds) for r in res[: len(systems)]]
    return xs, infos


def gmres(g_block, chi, b, chi_scale=1.0, device=0, **kw):
    """One-shot solve: builds a Solver, sets the operator and solves."""
    with Solver(device) as s:
        s.set_operator(g_block, chi, chi_scale)
        return s.solve(b, **kw)


# ---------------------------------------------------------------- PyGMRES API
def get_plane_wave(k, size):
    """exp(-i k col) on a size x size grid (PyGMRES/GMRES.py:13-18, angle 0)."""
    y, x = np.mgrid[:size, :size]
    return np.exp(-1j * k * x)


def get_green_matrix(k, size):
    """g[j_row, i_col] = (i/4) H0(k sqrt((i - 1/2)^2 + j^2)) (PyGMRES/GMRES.py:23-27)."""
    return green_block("pygmres", size, k)


def get_toeplitz_mat(ij_block):
    """Even (2N-1)^2 circulant of an N x N block (PyGMRES/GMRES.py:64-69)."""
    b = np.asarray(ij_block)
    t1 = np.hstack((b, b[:, :0:-1]))
    t2 = np.hstack((b[:0:-1, :], b[:0:-1, :0:-1]))
    return np.vstack((t1, t2))


def get_eps_from_mask(e, mask):
    """(e - 1) * mask as an (N^2, 1) column (PyGMRES/GMRES.py:60-61)."""
    return (e - 1) * np.asarray(mask).reshape((-1, 1))


_mv_cache = {}


def matvec(x, eps, k, qweq=False, transpose=False, g=None, device=0):
    """x - G (k^2 eps x) on the GPU, the reference's matvec(x, eps, k)
    (PyGMRES/GMRES.py:47-57).  x: N^2 vector, eps: N^2 real column, k: wavenumber,
    g: optional (2N-1)^2 circulant (as get_toeplitz_mat returns).  Returns an
    (N^2, 1) complex128 column.  ``qweq`` returns (G_block, G) as the reference;
    ``transpose`` gives x - chi G x (k^2 eps = chi), the reference's transposed
    operator."""
    x = np.asarray(x).reshape(-1)
    n = x.size
    N = int(round(np.sqrt(n)))
    if N * N != n:
        raise ValueError("x must hold N^2 entries")
    if g is None:
        block = get_green_matrix(k, N)
    else:
        block = np.asarray(g)[:N, :N]
    if qweq:
        return block, (get_toeplitz_mat(block) if g is None else g)
    chi = np.asarray(eps, dtype=np.float64).reshape(N, N)
    key = (device, N)
    s = _mv_cache.get(key)
    if s is None:
        s = Solver(device)
        _mv_cache[key] = s
    s.set_operator(block, chi, float(k) ** 2)
    return s.matvec(x.reshape(N, N).astype(np.complex128), transpose=transpose).reshape(-1, 1)


def fast_gmres(g_prep, mask, solution, maxiter, tolerance, chi_value, rhs=None, precision="fp64"):
    """The reference's Fast_GMRES_with_CUDA semantics (CUDA_GMRES/GMRES.cuh:22-446)
    through cugmres_fast_gmres.  Returns (solution complex64 N x N,
    actual_residual[maxiter+1] float32, GMRES_n, res_vs_tol)."""
    g_prep = np.ascontiguousarray(g_prep, np.complex64)
    N = (g_prep.shape[0] + 1) // 2
    m = np.ascontiguousarray(np.asarray(mask).reshape(N, N), np.uint8)
    sol = np.array(solution, dtype=np.complex64, order="C", copy=True).reshape(N, N)
    res = np.zeros(int(maxiter) + 1, np.float32)
    n = ctypes.c_uint(0)
    flag = ctypes.c_int(0)
    rp = None
    if rhs is not None:
        rhs = np.ascontiguousarray(rhs, np.complex64)
        rp = rhs.ctypes.data_as(ctypes.c_void_p)
    check(_lib.lib().cugmres_fast_gmres(
        g_prep.ctypes.data_as(ctypes.c_void_p), m.ctypes.data_as(ctypes.c_void_p),
        sol.ctypes.data_as(ctypes.c_void_p), res.ctypes.data_as(ctypes.c_void_p), ctypes.byref(n),
        ctypes.c_float(tolerance), ctypes.byref(flag), ctypes.c_uint(int(maxiter)), ctypes.c_uint(N),
        ctypes.c_float(chi_value), rp, _PREC[precision]), "cugmres_fast_gmres")
    return sol, res, n.value, bool(flag.value)
