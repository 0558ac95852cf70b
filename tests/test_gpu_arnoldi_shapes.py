"""Every launch shape of the two DCGS2 streaming passes (dot pass and axpy
pass, selected with CUGMRES_DOTS2_SHAPE / CUGMRES_AXPY2_SHAPE) gives the same
solve as the default shapes: group-major, tile-major (8, 7, 16 and 14 points
per lane; FP32 also on 16-byte pairs of complex values) and split kernels, on
grids whose size is not a multiple of any tile (n = 96^2, 97^2 (odd: the
FP32 pair shapes fall back to single values) and 150^2), in FP64 and mixed
precision."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import cugmres_b200 as cg
from cugmres_b200 import problems as P
out = {}
for N, eps in ((96, 2.0), (97, 2.0), (150, 2.0)):
    pr = P.helmholtz(N, eps, seed=N)
    s = cg.Solver(0).set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    for prec in ("fp64", "mixed"):
        x, info = s.solve(pr["b"], restart=60, max_iter=3000, tol=1e-10, precision=prec)
        assert info["status"] == 0, (N, prec, info["status_text"])
        out[f"x_{N}_{prec}"] = x
        out[f"it_{N}_{prec}"] = info["iterations"]
        out[f"res_{N}_{prec}"] = info["rel_residual_true"]
    s.close()
np.savez(sys.argv[2], **out)
"""

DOTS = [str(v) for v in range(13)]
AXPY = [str(v) for v in range(11)]


def _run(tmp_path, name, env_extra):
    env = dict(os.environ)
    env["CUGMRES_TUNE_CACHE"] = str(tmp_path.parent / "tune_arnoldi_shapes.txt")
    env.update(env_extra)
    out = tmp_path / f"{name}.npz"
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT, str(out)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.load(out)


@pytest.fixture(scope="module")
def default_run(tmp_path_factory, cuda_device):
    return _run(tmp_path_factory.mktemp("default"), "default", {})


def _compare(got, ref):
    for N in (96, 97, 150):
        for prec in ("fp64", "mixed"):
            assert got[f"res_{N}_{prec}"] <= 1e-10
            assert abs(int(got[f"it_{N}_{prec}"]) - int(ref[f"it_{N}_{prec}"])) <= 1, (N, prec)
            x, xr = got[f"x_{N}_{prec}"], ref[f"x_{N}_{prec}"]
            # both solves converged to 1e-10; only the summation order differs
            assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-8, (N, prec)


@pytest.mark.parametrize("shape", DOTS)
def test_dot_pass_shape(default_run, tmp_path, shape):
    _compare(_run(tmp_path, f"dots{shape}", {"CUGMRES_DOTS2_SHAPE": shape}), default_run)


@pytest.mark.parametrize("shape", AXPY)
def test_axpy_pass_shape(default_run, tmp_path, shape):
    _compare(_run(tmp_path, f"axpy{shape}", {"CUGMRES_AXPY2_SHAPE": shape}), default_run)
