"""Restart lengths whose scratch arrays put a kernel's dynamic shared memory
just under 48 KB: with the kernel's static shared memory the launch needs the
opt-in above 48 KB, which the launchers once skipped because they compared the
dynamic size alone (delayed CGS2 failed to launch its step kernel at restarts
1067..1227; the s-step Hessenberg kernel at 756..759 with S = 4 and 368..375
with S = 8).  Each case runs in a fresh context, so the scratch capacity is
the restart itself, and must give the GMRES(100) solution (the 64^2 system
converges in fewer steps than either restart, so the iterates are the same)."""
import numpy as np
import pytest

import cugmres_b200 as cg
from cugmres_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ortho, sstep, restart", [("dcgs2", 4, 1067), ("dcgs2", 4, 1227), ("cgs2", 4, 1100),
                                                   ("sstep", 4, 757), ("sstep", 8, 370)])
def test_restart_near_the_shared_memory_opt_in(cuda_device, ortho, sstep, restart):
    pr = P.helmholtz(64, 4.0, seed=0)
    with cg.Solver(cuda_device) as ref:
        ref.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
        xr, ir = ref.solve(pr["b"], restart=100, max_iter=2000, tol=1e-10, ortho=ortho, sstep=sstep)
    with cg.Solver(cuda_device) as s:
        s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
        x, info = s.solve(pr["b"], restart=restart, max_iter=2000, tol=1e-10, ortho=ortho, sstep=sstep)
    assert ir["status"] == 0 and info["status"] == 0, (ir["status_text"], info["status_text"])
    # eight-step Newton blocks lose rank on this spectrum and end their cycles
    # early (measured: 280 steps in 7 cycles at either restart); the others
    # finish in one cycle
    assert info["iterations"] == ir["iterations"] and info["cycles"] == (ir["cycles"] if sstep == 8 else 1)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10
