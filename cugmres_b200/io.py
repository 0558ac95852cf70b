"""Fixture and result I/O in the reference's formats, plus a binary writer.

* ASCII arrays as the reference writes and reads them
  (CUDA_GMRES/saveGPU.cuh:7-100 write, :181-199 read): complex arrays one
  "re im" pair per line, real / integer / boolean arrays one value per line
  (booleans as 0 / 1), row-major N x N grids flattened.  These are the formats
  of the reference's fixtures (Release/input/G_prep_N.txt, cylinder_N.txt,
  analytical_solution_N.txt) and of its per-run dumps (output/*.txt).
* `save_results` / `load_results`: one compressed .npz per run instead of the
  reference's per-run text files.
* `refined_stats`, `step_durations`: the statistics of the reference's timing
  notebook ("[RPW] Timestamps & Speedups.ipynb", cells defining the refined
  mean): the mean over the samples within one standard deviation of the mean
  (the plain mean if there are none) and the full-set standard deviation;
  durations are differences of consecutive positive timestamps.
"""
import numpy as np


def read_complex_txt(path, count=None):
    """Complex array from lines "re im" (complex128; the reference stores complex64)."""
    vals = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if vals.shape[1] != 2:
        raise ValueError(f"{path}: expected two columns (re im), got {vals.shape[1]}")
    out = vals[:, 0] + 1j * vals[:, 1]
    if count is not None:
        if out.size < count:
            raise ValueError(f"{path}: {out.size} values, expected {count}")
        out = out[:count]
    return out


def write_complex_txt(path, a, digits=12):
    """Lines "re im" with `digits` significant digits (the reference's setprecision)."""
    a = np.asarray(a).reshape(-1)
    with open(path, "w") as f:
        for v in a:
            f.write(f"{v.real:.{digits}g} {v.imag:.{digits}g}\n")


def read_real_txt(path, dtype=np.float64):
    """One value per line."""
    return np.loadtxt(path, dtype=dtype, ndmin=1)


def write_real_txt(path, a, digits=12):
    a = np.asarray(a).reshape(-1)
    with open(path, "w") as f:
        for v in a:
            f.write(f"{v:.{digits}g}\n")


def read_mask_txt(path, N):
    """N x N boolean mask from one 0 / 1 per line (cylinder_N.txt)."""
    m = np.loadtxt(path, dtype=np.int64, ndmin=1)
    if m.size < N * N:
        raise ValueError(f"{path}: {m.size} values, expected {N * N}")
    return m[: N * N].reshape(N, N) != 0


def write_mask_txt(path, mask):
    m = np.asarray(mask).reshape(-1)
    with open(path, "w") as f:
        for v in m:
            f.write("1\n" if v else "0\n")


def read_grid(path, N, kind="complex"):
    """An N x N grid in the reference's text format ('complex', 'real' or 'mask')."""
    if kind == "complex":
        return read_complex_txt(path, N * N).reshape(N, N)
    if kind == "real":
        return read_real_txt(path)[: N * N].reshape(N, N)
    if kind == "mask":
        return read_mask_txt(path, N)
    raise ValueError(kind)


def save_results(path, **arrays):
    """All of a run's arrays and scalars in one compressed .npz."""
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in arrays.items()})


def load_results(path):
    with np.load(path, allow_pickle=False) as d:
        return {k: d[k] for k in d.files}


def refined_stats(samples):
    """(refined mean, standard deviation): the mean over samples with
    |x - mean| < std, or the plain mean when no sample is that close."""
    x = np.asarray(samples, dtype=np.float64).reshape(-1)
    if x.size == 0:
        raise ValueError("no samples")
    mean, std = float(np.mean(x)), float(np.std(x))
    close = std > np.abs(x - mean)
    return (float(np.mean(x[close])) if np.any(close) else mean), std


def step_durations(timestamps):
    """Differences of consecutive positive timestamps (zeros are unused slots)."""
    t = np.asarray(timestamps).reshape(-1)
    t = t[t > 0]
    return t[1:] - t[:-1]
