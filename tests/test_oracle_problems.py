"""The oracle's own construction of the benchmark systems (used by the CPU
reference arm, which must not load the product library) gives the product's
arrays: contrast and right-hand side bit for bit, Green's block to rounding."""
import numpy as np
import pytest

from cugmres_b200 import problems as P
from oracle import problems as OP


@pytest.mark.parametrize("N,eps,seed,lh", [(32, 4.0, 0, 20.0), (96, 2.25, 7, 15.5), (130, 12.25, 3, 30.0)])
def test_oracle_problem_matches_product(oracle, N, eps, seed, lh):
    a = P.helmholtz(N, eps, seed=seed, cells_per_wavelength=lh)
    b = OP.helmholtz(N, eps, seed=seed, cells_per_wavelength=lh)
    assert np.array_equal(a["chi"], b["chi"])
    assert np.array_equal(a["b"], b["b"])
    assert a["k0"] == b["k0"] and a["h"] == b["h"] and a["chi_scale"] == b["chi_scale"]
    assert np.abs(a["g_block"] - b["g_block"]).max() <= 1e-15 * np.abs(b["g_block"]).max()


def test_embedding_size():
    for N, L in ((1, 16), (8, 16), (9, 32), (64, 128), (65, 256), (1024, 2048), (2048, 4096), (1100, 4096)):
        assert OP.embedding(N) == L
