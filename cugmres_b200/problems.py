"""Host-side construction of solver inputs (plain NumPy; no GPU work).

Two families:

* ``reference_cylinder(N)`` -- the reference's benchmark system: the
  dielectric cylinder of CUDA_GMRES/Release/input/cylinder_N.txt (centre row
  N/3, column N/2, radius N/6), wavenumber k = 2*3.14f/(N/6.f), contrast
  CHI = (2.25 - 1) k^2 (CUDA_GMRES/GMRES_kernels.cuh:12-19) and incident field
  exp(-i k row) used as right-hand side and initial guess
  (CUDA_GMRES/GMRES_kernels.cuh:557-572, launch_GMRES.cuh:158).
* ``helmholtz(N, eps_r, seed, ...)`` -- the GFIEM system A = I - k0^2 G diag(chi)
  on a grid of cell size h = wavelength / cells_per_wavelength: chi = eps_r - 1
  wherever a seeded Gaussian random field (white noise smoothed by a Gaussian
  of standard deviation `corr` cells, periodic, via FFT) is positive inside the
  central square of side fraction `fill`, chi = 0 elsewhere; b = exp(i k0 x),
  x = (row + 1/2) h on cell centres.

Arrays use the C convention of the reference's CUDA/MKL code: [row, col],
row-major, the row index being the axis of the reference Green's function's
half-cell offset.
"""
import ctypes

import numpy as np

from . import _lib


def green_block(kind, N, k0=0.0, h=0.0):
    """g[d1, d2] of the symmetric BTTB Green's matrix (host C++ via the C-ABI)."""
    kinds = {"helmholtz": _lib.CG_GREEN_HELMHOLTZ, "reference": _lib.CG_GREEN_REFERENCE,
             "pygmres": _lib.CG_GREEN_PYGMRES}
    kind = kinds.get(kind, kind)
    out = np.empty((N, N), np.complex128)
    _lib.check(_lib.lib().cugmres_green_block(int(kind), int(N), float(k0), float(h),
                                               out.ctypes.data_as(ctypes.c_void_p)), "green_block")
    return out


def reference_wavenumber(N):
    """k = 2*3.14f/(N/6.f) evaluated in float as the reference's macro."""
    return np.float32(np.float32(2 * 3.14) / np.float32(np.float32(N) / np.float32(6.0)))


def cylinder_mask(N):
    """Mask of cylinder_N.txt: (row - N/3)^2 + (col - N/2)^2 <= (N/6)^2."""
    r, c = np.mgrid[0:N, 0:N]
    return (r - N / 3) ** 2 + (c - N / 2) ** 2 <= (N / 6) ** 2


def reference_plane_wave(N):
    """exp(-i k row) rounded as the reference's complex8 incident field."""
    k = reference_wavenumber(N)
    arg = (-(np.float64(k)) * np.arange(N, dtype=np.float64)).astype(np.float32)
    row = (np.cos(arg.astype(np.float64)) + 1j * np.sin(arg.astype(np.float64))).astype(np.complex64)
    return np.repeat(row[:, None], N, axis=1).astype(np.complex128)


def reference_cylinder(N, eps=2.25):
    k = reference_wavenumber(N)
    chi_val = np.float32((np.float32(eps) - np.float32(1)) * k * k)
    mask = cylinder_mask(N)
    chi = np.where(mask, np.float64(chi_val), 0.0)
    b = reference_plane_wave(N)
    return dict(N=N, k=float(k), chi_value=float(chi_val), mask=mask, chi=chi, chi_scale=1.0,
                g_block=green_block("reference", N), b=b, x0=b.copy())


def gaussian_field(N, seed, corr=4.0):
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((N, N))
    f = np.fft.fftfreq(N)
    filt = np.exp(-2.0 * (np.pi * corr) ** 2 * (f[:, None] ** 2 + f[None, :] ** 2))
    return np.real(np.fft.ifft2(np.fft.fft2(w) * filt))


def sweep(nsys=256, seed=0, sides=(96, 128, 192, 256, 384, 512), lam_over_h=(15.0, 30.0), eps_range=(2.0, 12.0),
          with_green=True):
    """Seeded sweep of independent systems: grid side drawn from `sides`,
    wavelength / cell size uniform in `lam_over_h`, eps_r uniform in
    `eps_range`, one design seed each (the same field construction)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nsys):
        N = int(rng.choice(sides))
        lh = float(rng.uniform(*lam_over_h))
        eps = float(rng.uniform(*eps_range))
        out.append(helmholtz(N, eps, seed=int(rng.integers(1 << 30)), cells_per_wavelength=lh,
                             with_green=with_green))
    return out


def helmholtz(N, eps_r, seed=0, cells_per_wavelength=20.0, wavelength=1.0, corr=4.0, fill=0.75, with_green=True):
    """with_green=False leaves out the host-built g_block (Solver.set_operator_green
    and solve_batch build it on the GPU from k0 and h)."""
    k0 = 2.0 * np.pi / wavelength
    h = wavelength / cells_per_wavelength
    fld = gaussian_field(N, seed, corr)
    lo = int(round(N * (1.0 - fill) / 2.0))
    inside = np.zeros((N, N), bool)
    inside[lo:N - lo, lo:N - lo] = True
    chi = np.where(inside & (fld > 0), float(eps_r) - 1.0, 0.0)
    x = (np.arange(N) + 0.5) * h
    b = np.repeat(np.exp(1j * k0 * x)[:, None], N, axis=1)
    out = dict(N=N, k0=k0, h=h, eps_r=float(eps_r), seed=seed, chi=chi, chi_scale=k0 * k0, b=b)
    if with_green:
        out["g_block"] = green_block("helmholtz", N, k0, h)
    return out
