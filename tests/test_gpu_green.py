"""Operator set-up on the GPU: the device Green's block against the host
construction, and solves with the device-built operator."""
import ctypes

import numpy as np
import pytest

import cugmres_b200 as cg
from cugmres_b200 import _lib, problems as P

pytestmark = pytest.mark.gpu


def _device_block(kind, N, k0, h):
    import torch
    out = torch.empty((N, N), dtype=torch.complex128, device="cuda")
    kinds = {"helmholtz": 0, "reference": 1, "pygmres": 2}
    st = _lib.lib().cugmres_green_block_device(kinds[kind], N, k0, h, ctypes.c_void_p(out.data_ptr()), None)
    assert st == 0, _lib.strerror(st)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("kind,N,k0,h", [("helmholtz", 64, 2 * np.pi, 0.05), ("helmholtz", 300, 2 * np.pi, 1 / 15),
                                         ("pygmres", 48, 1.3, 0.0), ("reference", 64, 0.0, 0.0)])
def test_device_green_block_matches_host(cuda_device, kind, N, k0, h):
    g_dev = _device_block(kind, N, k0, h)
    g_host = P.green_block(kind, N, k0, h)
    err = np.abs(g_dev - g_host).max() / np.abs(g_host).max()
    # CUDA's and the host library's double-precision Bessel functions differ in the last bits;
    # the reference kind is rounded to complex64 on both sides
    assert err < (1e-7 if kind == "reference" else 1e-12), err


def test_solve_with_device_operator(cuda_device):
    pr = P.helmholtz(128, 4.0, seed=3)
    a, b = cg.Solver(0), cg.Solver(0)
    a.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    b.set_operator_green(128, pr["chi"], pr["chi_scale"], k0=pr["k0"], h=pr["h"])
    xa, ia = a.solve(pr["b"], restart=200, max_iter=3000, tol=1e-10)
    xb, ib = b.solve(pr["b"], restart=200, max_iter=3000, tol=1e-10)
    assert ia["status"] == 0 and ib["status"] == 0 and ib["rel_residual_true"] <= 1e-10
    assert abs(ia["iterations"] - ib["iterations"]) <= 1
    assert np.linalg.norm(xa - xb) / np.linalg.norm(xa) < 1e-8
    a.close()
    b.close()


def test_batch_with_device_green(cuda_device):
    """Device-built operators give the same batch results as host-built blocks."""
    systems = P.sweep(nsys=6, seed=4, sides=(96, 128), eps_range=(2.0, 4.0))
    xa, ia = cg.solve_batch(systems, workers=3, restart=100, max_iter=4000, tol=1e-10)
    xb, ib = cg.solve_batch(systems, workers=3, restart=100, max_iter=4000, tol=1e-10, device_green=True)
    for a, b, x1, x2 in zip(ia, ib, xa, xb):
        assert a["status"] == 0 and b["status"] == 0 and b["rel_residual_true"] <= 1e-10
        assert abs(a["iterations"] - b["iterations"]) <= 1
        assert np.linalg.norm(x1 - x2) / np.linalg.norm(x1) < 1e-8
