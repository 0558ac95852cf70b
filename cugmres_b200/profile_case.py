"""Deterministic launch sequence for profiler captures of the solver kernels.

    python -m cugmres_b200.profile_case [N] [--steps S] [--precision fp64|mixed]

builds the seeded Helmholtz system helmholtz(N, eps_r=4, seed=0) (N=1024 by
default: a 2048 x 2048 embedding, about 0.6 GB on the device), applies the
operator three times in FP64 and three times in FP32, then runs one
unrestarted solve of exactly S Arnoldi steps (default 60, tolerance 1e-14 so
it never stops early).  The launch order is therefore fixed:

    set-up (embedding FFTs, autotuner trials)
    3 x FP64 matvec   = 3 x [k_rows_forward, k_cols_convolve, k_rows_inverse]
    3 x FP32 matvec
    solve: residual, cycle start, then per step
           [rows_forward, cols_convolve, rows_inverse, k_dots2, k_dcgs2_step, k_axpy2]

so `ncu -k regex:k_dots2 -s 30 -c 1` picks the dot pass of step 30, and
`-k regex:"k_(rows_forward|cols_convolve|rows_inverse)" -s 3 -c 3` the passes
of the second FP64 matvec after the autotuner (the tuner's own trial
launches come first, so the number to skip depends on whether its on-disk
cache is warm; set CUGMRES_AUTOTUNE=0 for a fixed count).
"""
import argparse

import numpy as np

from . import Solver
from . import problems


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("N", type=int, nargs="?", default=1024)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--precision", default="fp64", choices=("fp64", "mixed"))
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    pr = problems.helmholtz(a.N, 4.0, seed=0)
    s = Solver(a.device)
    s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = np.random.default_rng(0).standard_normal((a.N, a.N)) + 0j
    for _ in range(3):
        s.matvec(x)
    x32 = x.astype(np.complex64)
    for _ in range(3):
        s.matvec(x32, precision="fp32")
    _, info = s.solve(pr["b"], restart=a.steps, max_iter=a.steps, tol=1e-14, precision=a.precision)
    print("ok", info["iterations"], info["status_text"])


if __name__ == "__main__":
    main()
