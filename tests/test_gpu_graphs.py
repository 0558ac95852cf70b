"""The restart cycle replayed as a CUDA graph gives the same iterates as
direct launches (bitwise), including a budget that ends inside a cycle."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CODE = r'''
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import cugmres_b200 as cg
from cugmres_b200 import problems as P
out = {}
for N, prec, ortho, m, maxit in ((96, "fp64", "dcgs2", 40, 130), (96, "mixed", "dcgs2", 40, 130),
                                 (64, "fp64", "cgs2", 30, 95), (128, "fp64", "dcgs2", 500, 120)):
    pr = P.helmholtz(N, 4.0, seed=7)
    s = cg.Solver(0)
    s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    x, info = s.solve(pr["b"], restart=m, max_iter=maxit, tol=1e-13, precision=prec, ortho=ortho)
    x2, info2 = s.solve(pr["b"], restart=m, max_iter=maxit, tol=1e-13, precision=prec, ortho=ortho)
    out[f"{N}_{prec}_{ortho}"] = (x, info["iterations"], info["res_hist"], x2)
    s.close()
np.savez(sys.argv[2], **{k + "_x": v[0] for k, v in out.items()}, **{k + "_it": v[1] for k, v in out.items()},
         **{k + "_h": v[2] for k, v in out.items()}, **{k + "_x2": v[3] for k, v in out.items()})
'''


def _run(tmp_path, graphs):
    f = str(tmp_path / f"g{graphs}.npz")
    env = dict(os.environ, CUGMRES_GRAPHS=str(graphs))
    r = subprocess.run([sys.executable, "-c", CODE, ROOT, f], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(f)


def test_graph_replay_matches_direct_launches(tmp_path):
    a = _run(tmp_path, 1)
    b = _run(tmp_path, 0)
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k
    # replaying the cached graph a second time gives the same result again
    for k in [f for f in a.files if f.endswith("_x")]:
        assert np.array_equal(a[k], a[k + "2"]), k
