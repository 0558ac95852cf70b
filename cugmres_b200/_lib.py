"""ctypes bindings of include/cugmres.h (libcugmres.so, built in-tree).

The library is loaded from cugmres_b200/lib/libcugmres.so.  There is no CPU
fallback: if the library is missing or cannot be loaded, every call raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcugmres.so")

CG_OK = 0
CG_ERR_INVALID = 1
CG_ERR_CUDA = 2
CG_ERR_NOT_CONVERGED = 3
CG_ERR_BREAKDOWN = 4
CG_ERR_NONFINITE = 5
CG_ERR_TIMEOUT = 6
CG_ERR_NOT_IMPLEMENTED = 7
CG_ERR_NO_OPERATOR = 8
CG_ERR_OOM = 9

CG_PREC_FP64 = 0
CG_PREC_MIXED = 1
CG_GIVENS_UNITARY = 0
CG_ORTHO_DCGS2 = 0
CG_ORTHO_CGS2 = 1
CG_ORTHO_SSTEP = 2
CG_GIVENS_REFERENCE = 1
CG_GREEN_HELMHOLTZ = 0
CG_GREEN_REFERENCE = 1
CG_GREEN_PYGMRES = 2
NOALLOC_MAX_N = 256

# Every symbol include/cugmres.h declares.
EXPORTS = (
    "cugmres_strerror", "cugmres_version", "cugmres_default_opts", "cugmres_create", "cugmres_destroy",
    "cugmres_set_stream", "cugmres_synchronize", "cugmres_green_block", "cugmres_set_operator",
    "cugmres_set_operator_circulant", "cugmres_grid_size", "cugmres_matvec", "cugmres_residual",
    "cugmres_solve", "cugmres_fast_gmres", "cugmres_profile", "cugmres_profile_read", "cugmres_matvec_noalloc",
    "cugmres_matvec_shapes", "cugmres_solve_batch", "cugmres_fno_create", "cugmres_fno_destroy",
    "cugmres_fno_info", "cugmres_fno_get_params", "cugmres_fno_set_params", "cugmres_fno_forward",
    "cugmres_fno_loss_grad", "cugmres_fno_train_step", "cugmres_set_preconditioner", "cugmres_gemm_bf16",
    "cugmres_matvec_transpose", "cugmres_fno_forward_train", "cugmres_fno_backward", "cugmres_fno_set_local_last",
    "cugmres_set_operator_green", "cugmres_green_block_device", "cugmres_solve_buckets",
)

PHASES = ("matvec", "dots", "axpy", "small", "update", "residual", "precond")


class CgOpts(ctypes.Structure):
    _fields_ = [
        ("restart", ctypes.c_int),
        ("max_iter", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("givens", ctypes.c_int),
        ("inner_tol", ctypes.c_double),
        ("zero_x0", ctypes.c_int),
        ("fixed_iterations", ctypes.c_int),
        ("timeout_s", ctypes.c_double),
        ("ortho", ctypes.c_int),
        ("preconditioner", ctypes.c_int),
        ("learned_x0", ctypes.c_int),
        ("transpose", ctypes.c_int),
        ("sstep", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
    ]


class CgResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("cycles", ctypes.c_int),
        ("rel_residual_estimate", ctypes.c_double),
        ("rel_residual_true", ctypes.c_double),
        ("seconds", ctypes.c_double),
        ("preconditioned_cycles", ctypes.c_int),
        ("x0_learned", ctypes.c_int),
    ]


class CgFnoInfo(ctypes.Structure):
    _fields_ = [
        ("layers", ctypes.c_int),
        ("width", ctypes.c_int),
        ("modes1", ctypes.c_int),
        ("modes2", ctypes.c_int),
        ("hidden", ctypes.c_int),
        ("in_features", ctypes.c_int),
        ("num_params", ctypes.c_longlong),
        ("steps", ctypes.c_longlong),
    ]


class CgSystem(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int),
        ("g_block", ctypes.c_void_p),
        ("chi", ctypes.c_void_p),
        ("chi_scale", ctypes.c_double),
        ("b", ctypes.c_void_p),
        ("x", ctypes.c_void_p),
        ("k0", ctypes.c_double),
        ("h", ctypes.c_double),
    ]


class CgPhaseStats(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double), ("bytes", ctypes.c_double), ("launches", ctypes.c_longlong)]


class CugmresError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = strerror(status)
        super().__init__(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")


_lib = None


def lib():
    """Loads libcugmres.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m cugmres_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L):
    P, I, D, F, U = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_uint
    L.cugmres_strerror.argtypes = [I]
    L.cugmres_strerror.restype = ctypes.c_char_p
    L.cugmres_version.restype = I
    L.cugmres_default_opts.argtypes = [ctypes.POINTER(CgOpts)]
    L.cugmres_default_opts.restype = None
    L.cugmres_create.argtypes = [ctypes.POINTER(P), I]
    L.cugmres_destroy.argtypes = [P]
    L.cugmres_set_stream.argtypes = [P, P]
    L.cugmres_synchronize.argtypes = [P]
    L.cugmres_green_block.argtypes = [I, I, D, D, P]
    L.cugmres_set_operator.argtypes = [P, I, P, P, D]
    L.cugmres_set_operator_circulant.argtypes = [P, I, P, P, D]
    L.cugmres_set_operator_green.argtypes = [P, I, I, D, D, P, D]
    L.cugmres_green_block_device.argtypes = [I, I, D, D, P, P]
    L.cugmres_grid_size.argtypes = [P, ctypes.POINTER(I), ctypes.POINTER(I)]
    L.cugmres_matvec.argtypes = [P, P, P, I]
    L.cugmres_matvec_transpose.argtypes = [P, P, P, I]
    L.cugmres_residual.argtypes = [P, P, P, P, ctypes.POINTER(D)]
    L.cugmres_solve.argtypes = [P, P, P, ctypes.POINTER(CgOpts), P, I, ctypes.POINTER(CgResult)]
    L.cugmres_fast_gmres.argtypes = [P, P, P, P, ctypes.POINTER(U), F, ctypes.POINTER(I), U, U, F, P, I]
    L.cugmres_matvec_noalloc.argtypes = [I, P, P, D, P, P, P]
    L.cugmres_matvec_shapes.argtypes = [P, I, ctypes.POINTER(I)]
    L.cugmres_solve_batch.argtypes = [I, I, ctypes.POINTER(CgSystem), ctypes.POINTER(CgOpts), I,
                                      ctypes.POINTER(CgResult)]
    L.cugmres_solve_buckets.argtypes = [I, I, ctypes.POINTER(CgSystem), ctypes.POINTER(CgOpts), I,
                                        ctypes.POINTER(CgResult)]
    L.cugmres_profile.argtypes = [P, I]
    L.cugmres_profile_read.argtypes = [P, ctypes.POINTER(CgPhaseStats)]
    LL, ULL = ctypes.c_longlong, ctypes.c_ulonglong
    L.cugmres_fno_create.argtypes = [ctypes.POINTER(P), I, ULL]
    L.cugmres_fno_destroy.argtypes = [P]
    L.cugmres_fno_destroy.restype = None
    L.cugmres_fno_info.argtypes = [P, ctypes.POINTER(CgFnoInfo)]
    L.cugmres_fno_get_params.argtypes = [P, P]
    L.cugmres_fno_set_params.argtypes = [P, P]
    L.cugmres_fno_forward.argtypes = [P, I, I, I, P, P, P, P]
    L.cugmres_fno_loss_grad.argtypes = [P, I, I, I, P, P, P, P, ctypes.POINTER(F), P]
    L.cugmres_fno_train_step.argtypes = [P, I, I, I, P, P, P, P, F, ctypes.POINTER(F)]
    L.cugmres_set_preconditioner.argtypes = [P, P, D]
    L.cugmres_fno_forward_train.argtypes = [P, I, I, I, P, P, P, P]
    L.cugmres_fno_backward.argtypes = [P, P, P, F]
    L.cugmres_fno_set_local_last.argtypes = [P, I]
    L.cugmres_gemm_bf16.argtypes = [I, LL, I, I, P, P, P]
    for name in EXPORTS:
        if name not in ("cugmres_strerror", "cugmres_default_opts", "cugmres_fno_destroy"):
            getattr(L, name).restype = I


def strerror(status):
    try:
        return lib().cugmres_strerror(int(status)).decode()
    except Exception:
        return "unknown"


def check(status, what=""):
    if status != CG_OK:
        raise CugmresError(status, what)
    return status
