"""Generate the golden fixtures under tests/golden/ from the reference checkout.

Run once, in a container that has the reference checkout mounted; ``--ref``
(required) is the directory that holds the reference project's top folder:

    python tests/golden/make_golden.py --ref <reference checkout>

Nothing at test time reads the reference checkout; the tests read only the
``.npz`` / ``.json`` files this script writes.  What is extracted and why:

* ``ref_mkl_solution_256_m44.npz`` -- the complex64 solution written by the
  reference's MKL GMRES for N=256, maxiter=44, x0 = b = plane wave, cylinder
  mask (MKL_GMRES_test_09122019/_results/test_residuals/solution_256_4400.txt,
  produced by MKL_GMRES_test_09122019/source/main.cpp:35-72), plus its
  residual estimate (residual_256_4400.txt) and wall time (time_256_4400.txt).
* ``ref_G_prep_{32,64}.npz`` -- the spatial (2N-1)x(2N-1) circulant of Green's
  function samples the CUDA driver reads (CUDA_GMRES/Release/input/G_prep_N.txt,
  read by CUDA_GMRES/launch_GMRES.cuh:70-77 via saveGPU.cuh:181-199).
* ``ref_cylinder_{32,64,256}.npz`` -- the 0/1 scatterer masks
  (CUDA_GMRES/Release/input/cylinder_N.txt, read by launch_GMRES.cuh:55-68).
* ``ref_analytical_{64,256}.npz`` -- Mie-series fields the reference compares
  against (CUDA_GMRES/Release/input/analytical_solution_N.txt,
  launch_GMRES.cuh:197-218).
* ``ref_results.json`` -- the published relative-error and residual histories
  (Results/relative_errors_256_0.npy, Results/residuals_256_0.npy).
* ``pygmres_matvec.npz`` -- outputs of the reference's own NumPy functions
  ``get_green_matrix``, ``get_toeplitz_mat`` and ``matvec`` (also with
  ``transpose=True``) (PyGMRES/GMRES.py:23-69)
  on seeded inputs.  Only the function definitions of GMRES.py are executed;
  its module-level benchmark loop (GMRES.py:95-221) is skipped.
"""
import argparse
import ast
import json
import os

import numpy as np

SUB = ("Benchmarks of CUDA-based GMRES Solver for Toeplitz and Hankel Matrices "
       "and Applications to Topology Optimization of Photonic Devices")
HERE = os.path.dirname(os.path.abspath(__file__))


def load_complex_txt(path):
    a = np.loadtxt(path, dtype=np.float64)
    return (a[:, 0] + 1j * a[:, 1]).astype(np.complex64)


def load_mask_txt(path, n):
    with open(path) as f:
        bits = [c for c in f.read() if c in "01"]
    assert len(bits) == n * n, (path, len(bits))
    return np.array([c == "1" for c in bits], dtype=bool).reshape(n, n)


def load_pygmres_defs(path):
    """Execute only the imports and function definitions of PyGMRES/GMRES.py."""
    tree = ast.parse(open(path).read())
    keep = [n for n in tree.body
            if isinstance(n, (ast.Import, ast.ImportFrom, ast.FunctionDef))]
    mod = ast.Module(body=keep, type_ignores=[])
    ns = {}
    exec(compile(mod, path, "exec"), ns)
    return ns


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="reference checkout (holds the project folder)")
    args = ap.parse_args()
    base = os.path.join(args.ref, SUB)
    inp = os.path.join(base, "CUDA_GMRES", "Release", "input")
    mkl = os.path.join(base, "MKL_GMRES_test_09122019", "_results", "test_residuals")

    sol = load_complex_txt(os.path.join(mkl, "solution_256_4400.txt"))
    res = float(open(os.path.join(mkl, "residual_256_4400.txt")).read().split()[0])
    tim = float(open(os.path.join(mkl, "time_256_4400.txt")).read().split()[0])
    np.savez_compressed(os.path.join(HERE, "ref_mkl_solution_256_m44.npz"),
                        solution=sol.reshape(256, 256), residual_estimate=np.float64(res),
                        time_s=np.float64(tim), N=256, maxiter=44, tolerance=1e-8)

    for n in (32, 64):
        g = load_complex_txt(os.path.join(inp, f"G_prep_{n}.txt"))
        np.savez_compressed(os.path.join(HERE, f"ref_G_prep_{n}.npz"),
                            g_prep=g.reshape(2 * n - 1, 2 * n - 1), N=n)
    for n in (32, 64, 256):
        m = load_mask_txt(os.path.join(inp, f"cylinder_{n}.txt"), n)
        np.savez_compressed(os.path.join(HERE, f"ref_cylinder_{n}.npz"),
                            mask=np.packbits(m.ravel()), N=n)
    for n in (64, 256):
        a = load_complex_txt(os.path.join(inp, f"analytical_solution_{n}.txt"))
        np.savez_compressed(os.path.join(HERE, f"ref_analytical_{n}.npz"),
                            field=a.reshape(n, n), N=n)

    rel = np.load(os.path.join(base, "Results", "relative_errors_256_0.npy"))
    rsd = np.load(os.path.join(base, "Results", "residuals_256_0.npy"))
    with open(os.path.join(HERE, "ref_results.json"), "w") as f:
        json.dump({"relative_errors_256": [float(v) for v in rel],
                   "residuals_256": [float(v) for v in rsd]}, f, indent=1)

    # The reference's own NumPy matvec on seeded inputs.
    ns = load_pygmres_defs(os.path.join(base, "PyGMRES", "GMRES.py"))
    rng = np.random.default_rng(1234)
    out = {}
    for n in (8, 16, 32):
        k = 2 * 3.14 / (n / 6)
        x = (rng.standard_normal(n * n) + 1j * rng.standard_normal(n * n))
        eps = (rng.random((n * n, 1)) < 0.4).astype(np.float64) * 1.25
        y = ns["matvec"](x, eps, k)
        yt = ns["matvec"](x, eps, k, transpose=True)
        gb = ns["get_green_matrix"](k, n)
        gt = ns["get_toeplitz_mat"](gb)
        out[f"x_{n}"] = x
        out[f"eps_{n}"] = eps
        out[f"k_{n}"] = np.float64(k)
        out[f"y_{n}"] = np.asarray(y).reshape(-1)
        out[f"yt_{n}"] = np.asarray(yt).reshape(-1)
        out[f"green_block_{n}"] = gb
        out[f"toeplitz_{n}"] = gt
    np.savez_compressed(os.path.join(HERE, "pygmres_matvec.npz"), **out)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
