"""CPU checks of the learned preconditioner's oracle: the manual backward
pass (the order the GPU follows) against torch autograd, the parameter
layout, and the homogeneity M(a r) = a M(r) the flexible solver relies on."""
import numpy as np

from oracle import fno_oracle as FO


def _setup(seed=0, B=2, H=32, W=40):
    rng = np.random.default_rng(seed)
    p = (rng.uniform(-1, 1, FO.NPARAM) * 0.2).astype(np.float32)
    for l in range(FO.LAYERS):
        o = FO.off_r(l)
        p[o:o + FO.RSZ] = rng.uniform(-1, 1, FO.RSZ) * 4.0 / (FO.C * FO.C)
    chi = (rng.random((B, H, W)) > 0.5) * rng.uniform(1, 10, (B, 1, 1))
    k0h = rng.uniform(0.2, 0.4, B)
    r = (rng.standard_normal((B, H, W)) + 1j * rng.standard_normal((B, H, W))).astype(np.complex64)
    x = (r + 0.3 * (rng.standard_normal((B, H, W)) + 1j * rng.standard_normal((B, H, W)))).astype(np.complex64)
    return p, chi, k0h, r, x


import pytest


@pytest.mark.parametrize("local_last", [True, False])
def test_manual_backward_matches_autograd(local_last):
    p, chi, k0h, r, x = _setup()
    l1, g1 = FO.loss_grad(p, chi, k0h, r, x, bf16=False, local_last=local_last)
    l2, g2 = FO.loss_grad_autograd(p, chi, k0h, r, x, local_last=local_last)
    assert abs(l1 - l2) <= 1e-6 * abs(l2)
    assert np.linalg.norm(g1 - g2) <= 1e-5 * np.linalg.norm(g2)


def test_pack_unpack_roundtrip():
    p, *_ = _setup(1)
    assert np.array_equal(FO.pack(FO.unpack(p)), p)


def test_positive_homogeneity():
    p, chi, k0h, r, _ = _setup(2, B=1)
    z1 = FO.forward(p, chi, k0h, r, bf16=False)["z"].numpy()
    z2 = FO.forward(p, chi, k0h, 3.5 * r, bf16=False)["z"].numpy()
    assert np.linalg.norm(z2 - 3.5 * z1) <= 1e-5 * np.linalg.norm(z2)
