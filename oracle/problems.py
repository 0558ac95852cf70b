"""Inputs of the benchmark configurations, built without the product library.
TEST INFRASTRUCTURE ONLY.

The CPU reference arm of bench.py and the tests need the same seeded systems
the GPU solver sees, but must not load libcugmres.so to get them.  This module
states the configurations' construction once more with NumPy and the oracle's
own Green's block (or_green_block_helmholtz):

* a Gaussian random field: white noise from numpy.random.default_rng(seed),
  smoothed by a Gaussian of standard deviation `corr` cells (periodic, FFT);
* contrast chi = eps_r - 1 where the field is positive inside the central
  square of side fraction `fill`, 0 elsewhere;
* right-hand side b = exp(i k0 x), x = (row + 1/2) h on cell centres;
* k0 = 2 pi / wavelength, h = wavelength / cells_per_wavelength.

tests/test_oracle_problems.py checks that this gives the product's
cugmres_b200.problems.helmholtz arrays exactly (chi, b) and its Green's block
to rounding.
"""
import numpy as np

from . import oracle as O


def gaussian_field(N, seed, corr=4.0):
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((N, N))
    f = np.fft.fftfreq(N)
    filt = np.exp(-2.0 * (np.pi * corr) ** 2 * (f[:, None] ** 2 + f[None, :] ** 2))
    return np.real(np.fft.ifft2(np.fft.fft2(w) * filt))


def helmholtz(N, eps_r, seed=0, cells_per_wavelength=20.0, wavelength=1.0, corr=4.0, fill=0.75):
    k0 = 2.0 * np.pi / wavelength
    h = wavelength / cells_per_wavelength
    fld = gaussian_field(N, seed, corr)
    lo = int(round(N * (1.0 - fill) / 2.0))
    inside = np.zeros((N, N), bool)
    inside[lo:N - lo, lo:N - lo] = True
    chi = np.where(inside & (fld > 0), float(eps_r) - 1.0, 0.0)
    x = (np.arange(N) + 0.5) * h
    b = np.repeat(np.exp(1j * k0 * x)[:, None], N, axis=1)
    return dict(N=N, k0=k0, h=h, eps_r=float(eps_r), seed=seed, chi=chi, chi_scale=k0 * k0, b=b,
                g_block=O.green_block_helmholtz(N, k0, h))


def embedding(N):
    """Smallest power of two L >= 2N - 1 (at least 16): the product's embedding."""
    L = 16
    while L < 2 * N - 1:
        L *= 2
    return L
