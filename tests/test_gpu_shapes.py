"""Every matvec launch shape the autotuner may pick gives the same operator
(A in FP64 and FP32, and the transposed operator A^T), for embeddings L = 128
to 4096."""
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
from oracle import oracle as O
for N in (64, 128, 300, 512, 1024, 1100):
    pr = P.helmholtz(N, 4.0, seed=N)
    s = cg.Solver(0).set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x = np.random.default_rng(N).standard_normal((N, N)) + 1j
    y = s.matvec(x)
    yo = O.matvec(O.spectrum(pr["g_block"], s.L), pr["chi"] * pr["chi_scale"], x)
    e64 = np.abs(y - yo).max() / np.abs(yo).max()
    y32 = s.matvec(x.astype(np.complex64), precision="fp32")
    e32 = np.abs(y32 - yo).max() / np.abs(yo).max()
    yt = s.matvec(x, transpose=True)  # A^T: the contrast moves to the inverse row pass
    yto = O.matvec_transpose(O.spectrum(pr["g_block"], s.L), pr["chi"] * pr["chi_scale"], x)
    et = np.abs(yt - yto).max() / np.abs(yto).max()
    print(N, s.matvec_shapes("fp64"), s.matvec_shapes("fp32"), e64, e32, et)
    assert e64 < 1e-13 and e32 < 2e-6 and et < 1e-13, (e64, e32, et)
"""


@pytest.mark.parametrize("shape", ["0", "1", "2", "3", "4", "5", "6", "7", "8", "9", "tuned"])
def test_matvec_shape_parity(cuda_device, shape, tmp_path):
    env = dict(os.environ)
    env["CUGMRES_TUNE_CACHE"] = str(tmp_path / "tune.txt")
    if shape != "tuned":
        env["CUGMRES_MATVEC_SHAPE"] = shape
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    if shape == "tuned":
        assert os.path.exists(env["CUGMRES_TUNE_CACHE"])


CHAIN_SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import cugmres_b200 as cg
from cugmres_b200 import problems as P
from oracle import oracle as O
for N in (64, 300):
    pr = P.helmholtz(N, 2.25, seed=N)
    s = cg.Solver(0).set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    for prec, tol in (("fp64", 1e-9), ("mixed", 1e-4)):
        x, info = s.solve(pr["b"], restart=20, max_iter=60, tol=0.0, ortho="sstep", sstep=4, precision=prec)
        o = O.gmres(O.spectrum(pr["g_block"], s.L), pr["chi"] * pr["chi_scale"], pr["b"], restart=20, maxiter=60, tol=0.0)
        err = np.linalg.norm(x - o["x"]) / np.linalg.norm(o["x"])
        print(N, prec, s.matvec_shapes(prec), info["iterations"], err)
        assert info["iterations"] == 60 and err < tol, (N, prec, err)
"""


@pytest.mark.parametrize("shape", ["0", "1", "4", "7", "9", "tuned"])
def test_sstep_chain_under_each_row_shape(cuda_device, shape, tmp_path):
    """The s-step Newton chain fuses each inverse row pass with the next forward
    row pass (k_rows_inv_fwd, in the inverse pass's launch shape): three whole
    GMRES(20) cycles on 64^2 and 300^2 (odd rows: N < L/2) give the oracle's
    iterate under every row shape, in FP64 and in the complex64 cycles."""
    env = dict(os.environ)
    env["CUGMRES_TUNE_CACHE"] = str(tmp_path / "tune.txt")
    if shape != "tuned":
        env["CUGMRES_MATVEC_SHAPE"] = shape
    r = subprocess.run([sys.executable, "-c", CHAIN_SCRIPT, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
