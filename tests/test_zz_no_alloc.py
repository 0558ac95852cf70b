"""cugmres_matvec_noalloc: the operator application for callers that cannot
allocate device memory (a plug-in whose host application owns all GPU memory
through its own pool, or a loop that cannot pay cudaMalloc's implicit device
synchronisation).  Every call reuses the one scratch array compiled into the
library, so two calls in a row with different grids must each give the
oracle's y = A x, and the same y as the context-based cugmres_matvec.

This file is collected last so that a failure here never hides the results of
the other GPU tests; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import cugmres_b200 as cg
from cugmres_b200 import _lib
from cugmres_b200 import problems as P

pytestmark = pytest.mark.gpu


def _noalloc(N, g, chi, scale, x, y, stream):
    return _lib.lib().cugmres_matvec_noalloc(int(N), ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(chi.data_ptr()),
                                              float(scale), ctypes.c_void_p(x.data_ptr()),
                                              ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(stream))


@pytest.mark.parametrize("grids", [((256, 1), (200, 2)), ((64, 3), (256, 4))])
def test_noalloc_matvec_matches_oracle_and_context_matvec(cuda_device, oracle, grids):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row with different grids and data (N = 256 is the limit):
    # the second must not see anything the first left in the shared scratch
    for N, seed in grids:
        pr = P.helmholtz(N, 4.0, seed=seed)
        rng = np.random.default_rng(seed)
        xh = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
        g = torch.from_numpy(pr["g_block"]).cuda()
        chi = torch.from_numpy(pr["chi"]).cuda()
        x = torch.from_numpy(xh).cuda()
        y = torch.full_like(x, complex("nan"))
        assert _noalloc(N, g, chi, pr["chi_scale"], x, y, stream) == _lib.CG_OK
        torch.cuda.synchronize()
        got = y.cpu().numpy()
        assert np.isfinite(got).all()
        with cg.Solver(cuda_device) as s:
            s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
            ctx = s.matvec(xh)
            L = s.L
        yo = oracle.matvec(oracle.spectrum(pr["g_block"], L), pr["chi"] * pr["chi_scale"], xh)
        assert np.abs(got - yo).max() / np.abs(yo).max() < 1e-13
        assert np.abs(got - ctx).max() / np.abs(ctx).max() < 1e-13


def test_noalloc_rejects_what_it_cannot_hold(cuda_device):
    import torch
    N = _lib.NOALLOC_MAX_N + 1
    g = torch.zeros((N, N), dtype=torch.complex128, device="cuda")
    chi = torch.zeros((N, N), dtype=torch.float64, device="cuda")
    x = torch.zeros((N, N), dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    assert _noalloc(N, g, chi, 1.0, x, y, 0) == _lib.CG_ERR_INVALID
    xh = torch.zeros((8, 8), dtype=torch.complex128)  # host memory is refused too
    g8 = torch.zeros((8, 8), dtype=torch.complex128, device="cuda")
    c8 = torch.zeros((8, 8), dtype=torch.float64, device="cuda")
    assert _noalloc(8, g8, c8, 1.0, xh, xh, 0) == _lib.CG_ERR_INVALID


def test_noalloc_rejects_another_devices_memory(cuda_device):
    """Memory of another GPU is refused before anything is launched."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs a second GPU to hold the foreign buffer")
    with torch.cuda.device(0):
        g = torch.zeros((8, 8), dtype=torch.complex128, device="cuda:0")
        c = torch.zeros((8, 8), dtype=torch.float64, device="cuda:0")
        y = torch.zeros((8, 8), dtype=torch.complex128, device="cuda:0")
        foreign = torch.zeros((8, 8), dtype=torch.complex128, device="cuda:1")
        assert _noalloc(8, g, c, 1.0, foreign, y, 0) == _lib.CG_ERR_INVALID
