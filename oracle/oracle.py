"""ctypes front-end of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

The oracle is a plain-C restatement of the reference's CPU GMRES
(MKL_GMRES_test_09122019/source/MKL_GMRES.h:3-395 and loop_functions.h) with
its own FFT.  Only tests/, the smoke check and bench.py's CPU-baseline leg may
import this module; the product (cugmres_b200) never does.

Every array is C-contiguous numpy: complex128 / float64 for the ``_z`` family,
complex64 / float32 for the ``_c`` family.  Grid arrays are N x N row-major
with the reference's convention: the first index is the row i (the axis of the
Green's-function half-cell offset in the reference construction).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build(force=False):
    """Compile oracle/_build/liboracle.so with the committed Makefile."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_F = ctypes.c_float


def _declare(L):
    for sfx in ("z", "c"):
        getattr(L, f"or_fft2d_{sfx}").argtypes = [_I, _P, _I]
        getattr(L, f"or_spectrum_{sfx}").argtypes = [_I, _I, _P, _P]
        getattr(L, f"or_matvec_{sfx}").argtypes = [_I, _I, _P, _P, _P, _P, _P]
        f = getattr(L, f"or_gmres_reference_{sfx}")
        f.argtypes = [_I, _I, _P, _P, _P, _P, _I, _D if sfx == "z" else _F, _P, _P, _P]
        f.restype = _I
        f = getattr(L, f"or_gmres_{sfx}")
        f.argtypes = [_I, _I, _P, _P, _P, _P, _I, _I, _D, _I, _I, _P, _P, _P, _P]
        f.restype = _I
    L.or_green_block_reference.argtypes = [_I, _I, _P]
    L.or_green_block_helmholtz.argtypes = [_I, _D, _D, _P]
    L.or_gmres_ir.argtypes = [_I, _I, _P, _P, _P, _P, _I, _D, _D, _I, _I, _I,
                              _P, _P, _P, _P]
    L.or_gmres_ir.restype = _I
    L.or_num_threads.restype = _I
    L.or_set_num_threads.argtypes = [_I]


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _types(precision):
    if precision in ("c128", "z", np.complex128):
        return "z", np.complex128, np.float64
    if precision in ("c64", "c", np.complex64):
        return "c", np.complex64, np.float32
    raise ValueError(precision)


def set_threads(n):
    lib().or_set_num_threads(int(n))


def num_threads():
    return lib().or_num_threads()


def green_block_reference(N, round_to_float=True):
    """Reference Green's block g(i,j) (loop_functions.h:128-168), complex128."""
    g = np.empty((N, N), np.complex128)
    lib().or_green_block_reference(N, int(bool(round_to_float)), _ptr(g))
    return g


def green_block_helmholtz(N, k0, h):
    """GFIEM Green's block with the h^2 weight and the disk self term."""
    g = np.empty((N, N), np.complex128)
    lib().or_green_block_helmholtz(N, float(k0), float(h), _ptr(g))
    return g


def fft2d(a, sign=-1, precision="c128"):
    sfx, ct, _ = _types(precision)
    a = np.ascontiguousarray(a, dtype=ct).copy()
    getattr(lib(), f"or_fft2d_{sfx}")(a.shape[0], _ptr(a), int(sign))
    return a


def spectrum(g_block, L, precision="c128"):
    """FFT2 of the even circulant embedding of g_block into L x L."""
    sfx, ct, _ = _types(precision)
    g = np.ascontiguousarray(g_block, dtype=ct)
    out = np.empty((L, L), ct)
    getattr(lib(), f"or_spectrum_{sfx}")(g.shape[0], L, _ptr(g), _ptr(out))
    return out


def matvec(ghat, chi, x, b=None, precision="c128"):
    """A x = x - G (chi x), or with b given the residual b - A x."""
    sfx, ct, rt = _types(precision)
    ghat = np.ascontiguousarray(ghat, dtype=ct)
    chi = np.ascontiguousarray(chi, dtype=rt)
    x = np.ascontiguousarray(x, dtype=ct)
    N, L = x.shape[0], ghat.shape[0]
    y = np.empty_like(x)
    bp = None
    if b is not None:
        b = np.ascontiguousarray(b, dtype=ct)
        bp = _ptr(b)
    getattr(lib(), f"or_matvec_{sfx}")(N, L, _ptr(ghat), _ptr(chi), _ptr(x), bp, _ptr(y))
    return y


def matvec_transpose(ghat, chi, x, precision="c128"):
    """A^T x = x - chi G x (G symmetric): the transposed operator of the
    reference's PyGMRES matvec(..., transpose=True) (PyGMRES/GMRES.py:52-53)
    and of its CUDA gradient path (CUDA_GMRES/GMRES_kernels.cuh:305-326).
    Built from the forward restatement: G x = x - (x - G (1 x))."""
    x = np.asarray(x)
    gx = x - matvec(ghat, np.ones(x.shape), x, precision=precision)
    return x - np.asarray(chi) * gx


def gmres_reference(ghat, chi, b, x0, maxiter, tol, precision="c128"):
    """Step-for-step restatement of FFT_GMRES_with_MKL (fixed maxiter, MGS,
    explicit Givens accumulation, LU solve).  Returns (x, res_hist, n, res_vs_tol, info)."""
    sfx, ct, rt = _types(precision)
    ghat = np.ascontiguousarray(ghat, dtype=ct)
    chi = np.ascontiguousarray(chi, dtype=rt)
    b = np.ascontiguousarray(b, dtype=ct)
    x = np.ascontiguousarray(x0, dtype=ct).copy()
    res = np.zeros(maxiter + 1, rt)
    n = ctypes.c_int(0)
    flag = ctypes.c_int(0)
    info = getattr(lib(), f"or_gmres_reference_{sfx}")(
        x.shape[0], ghat.shape[0], _ptr(ghat), _ptr(chi), _ptr(b), _ptr(x), int(maxiter),
        float(tol), _ptr(res), ctypes.byref(n), ctypes.byref(flag))
    return x, res, n.value, bool(flag.value), info


def gmres(ghat, chi, b, x0=None, restart=100, maxiter=1000, tol=1e-10, ortho="mgs",
          rotation="unitary", precision="c128"):
    """Restarted GMRES(m) with early exit on the relative residual estimate.
    Returns dict(x, res_hist, iterations, cycles, true_res, status)."""
    sfx, ct, rt = _types(precision)
    ghat = np.ascontiguousarray(ghat, dtype=ct)
    chi = np.ascontiguousarray(chi, dtype=rt)
    b = np.ascontiguousarray(b, dtype=ct)
    x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, dtype=ct).copy()
    hist = np.zeros(maxiter + 1, np.float64)
    it, cyc, tr = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
    st = getattr(lib(), f"or_gmres_{sfx}")(
        x.shape[0], ghat.shape[0], _ptr(ghat), _ptr(chi), _ptr(b), _ptr(x), int(restart),
        int(maxiter), float(tol), {"mgs": 0, "cgs2": 1}[ortho],
        {"reference": 0, "unitary": 1}[rotation], _ptr(hist), ctypes.byref(it),
        ctypes.byref(cyc), ctypes.byref(tr))
    return dict(x=x, res_hist=hist[: it.value + 1], iterations=it.value, cycles=cyc.value,
                true_res=tr.value, status=st)


def gmres_ir(ghat, chi, b, x0=None, inner_restart=50, inner_tol=1e-5, tol=1e-10,
             max_outer=1000, max_inner_total=100000, rotation="unitary"):
    """Complex64-inner / complex128-outer GMRES with iterative refinement."""
    ghat = np.ascontiguousarray(ghat, dtype=np.complex128)
    chi = np.ascontiguousarray(chi, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.complex128).copy()
    hist = np.zeros(max_outer + 1, np.float64)
    o, tot, tr = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
    st = lib().or_gmres_ir(x.shape[0], ghat.shape[0], _ptr(ghat), _ptr(chi), _ptr(b), _ptr(x),
                           int(inner_restart), float(inner_tol), float(tol), int(max_outer),
                           int(max_inner_total), {"reference": 0, "unitary": 1}[rotation],
                           _ptr(hist), ctypes.byref(o), ctypes.byref(tot), ctypes.byref(tr))
    return dict(x=x, outer_hist=hist[: o.value + 1], outer=o.value, inner_total=tot.value,
                true_res=tr.value, status=st)
