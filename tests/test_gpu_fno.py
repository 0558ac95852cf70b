"""Learned preconditioner on the GPU: the tcgen05 GEMM, the network's
forward pass and gradients against the CPU oracle, training, and flexible
GMRES with the trained network (gain over plain GMRES, fallback)."""
import ctypes

import numpy as np
import pytest

from cugmres_b200 import _lib, learned, problems
from oracle import fno_oracle as FO

pytestmark = pytest.mark.gpu


def _bf16_bits(a):
    """float32 -> (BF16 bits as uint16, the rounded float32 values), round to nearest even."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r, (r.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("M,N,K", [(1000, 32, 32), (128 * 300, 32, 32), (777, 128, 32), (4096, 32, 128),
                                   (513, 128, 128)])
def test_tcgen05_gemm(cuda_device, M, N, K):
    rng = np.random.default_rng(M + N + K)
    a16, a = _bf16_bits(rng.standard_normal((M, K)).astype(np.float32))
    b16, b = _bf16_bits(rng.standard_normal((N, K)).astype(np.float32))
    c = np.empty((M, N), np.float32)
    st = _lib.lib().cugmres_gemm_bf16(0, M, N, K, a16.ctypes.data_as(ctypes.c_void_p),
                                      b16.ctypes.data_as(ctypes.c_void_p), c.ctypes.data_as(ctypes.c_void_p))
    assert st == 0, _lib.strerror(st)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    # BF16 x BF16 products are exact in FP32; only the FP32 accumulation order differs
    assert np.max(np.abs(c - ref)) <= 1e-5 * np.max(np.abs(ref)) + 1e-6


def _params(seed):
    """Random parameters with activations of order one (R larger than the default init)."""
    net_p = np.random.default_rng(seed)
    p = net_p.uniform(-1, 1, FO.NPARAM).astype(np.float32)
    p[FO.OFF_P:FO.OFF_L0] *= 0.5
    for l in range(FO.LAYERS):
        o = FO.off_r(l)
        p[o:o + FO.RSZ] *= 4.0 / (FO.C * FO.C)
        p[o + FO.RSZ:o + FO.LSZ] *= 1.0 / np.sqrt(FO.C)
    p[FO.OFF_Q1:FO.OFF_Q2] *= 1.0 / np.sqrt(FO.C)
    p[FO.OFF_Q2:] *= 1.0 / np.sqrt(FO.HID)
    return p


def _inputs(B, H, W, seed):
    rng = np.random.default_rng(seed)
    chi = ((rng.random((B, H, W)) > 0.5) * rng.uniform(1, 11, (B, 1, 1))).astype(np.float32)
    k0h = rng.uniform(0.2, 0.42, B).astype(np.float32)
    r = (rng.standard_normal((B, H, W)) + 1j * rng.standard_normal((B, H, W))).astype(np.complex64)
    x = (r + 0.5 * (rng.standard_normal((B, H, W)) + 1j * rng.standard_normal((B, H, W)))).astype(np.complex64)
    return chi, k0h, r, x


@pytest.fixture(scope="module")
def net(cuda_device):
    n = learned.FNO(0, seed=0)
    yield n
    n.close()


def test_fno_params_roundtrip(net):
    info = net.info()
    assert (info["layers"], info["width"], info["modes1"], info["modes2"], info["hidden"]) == (4, 32, 16, 16, 128)
    assert info["num_params"] == FO.NPARAM
    p = _params(3)
    net.set_params(p)
    assert np.array_equal(net.get_params(), p)


@pytest.mark.parametrize("B,H,W", [(2, 32, 48), (1, 64, 64), (3, 40, 96), (1, 32, 1024), (2, 40, 1024)])
def test_fno_forward_matches_oracle(net, B, H, W):
    """W = 1024 takes the tensor-core column DFT (two-level split, BF16 hi/lo
    twiddles), the other widths the CUDA-core one."""
    p = _params(1)
    net.set_params(p)
    chi, k0h, r, _ = _inputs(B, H, W, 7)
    z = net.forward(chi, k0h, r)
    ref = FO.forward(p, chi, k0h, r, bf16=True)
    s = ref["s"].numpy().reshape(-1, 1, 1)
    corr = (z - r) / s
    corr_ref = (ref["z"].numpy() - r) / s
    err = np.linalg.norm(corr - corr_ref) / np.linalg.norm(corr_ref)
    # BF16 storage of activations: isolated one-ulp differences propagate through 5 layers
    assert err < 2e-2, err


@pytest.mark.parametrize("local_last,shape", [(True, (2, 32, 40)), (False, (2, 32, 40)), (True, (1, 32, 1024))])
def test_fno_gradients_match_oracle(net, local_last, shape):
    """(1, 32, 1024): the width whose forward pass takes the tensor-core column
    DFTs (BF16 twiddles, BF16 Z in the inverse) while the backward pass runs the
    CUDA-core adjoint DFTs on what that forward saved."""
    p = _params(2)
    net.set_params(p)
    net.set_local_last(local_last)
    chi, k0h, r, x = _inputs(*shape, 11)
    loss, g = net.loss_grad(chi, k0h, r, x)
    net.set_local_last(True)
    loss_ref, g_ref = FO.loss_grad(p, chi, k0h, r, x, bf16=True, local_last=local_last)
    assert abs(loss - loss_ref) <= 5e-3 * abs(loss_ref), (loss, loss_ref)
    blocks = {"P": (FO.OFF_P, FO.OFF_L0), "Q1": (FO.OFF_Q1, FO.OFF_Q2), "Q2": (FO.OFF_Q2, FO.NPARAM)}
    for l in range(FO.LAYERS):
        o = FO.off_r(l)
        blocks[f"R{l}"] = (o, o + FO.RSZ)
        blocks[f"W{l}"] = (o + FO.RSZ, o + FO.LSZ)
    if not local_last:
        o = FO.off_r(FO.LAYERS - 1) + FO.RSZ
        assert np.all(g[o:o + FO.C * FO.C] == 0)
        blocks[f"W{FO.LAYERS - 1}"] = (o + FO.C * FO.C, o + FO.C * FO.C + FO.C)  # b_3 only
    for name, (a, b) in blocks.items():
        e = np.linalg.norm(g[a:b] - g_ref[a:b]) / np.linalg.norm(g_ref[a:b])
        # the oracle mirrors every BF16 rounding of the GPU; the rest is FP32 summation order
        assert e < 5e-2, (name, e)


_CUDA_CORE_SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from cugmres_b200 import learned
d = np.load(sys.argv[2])
n = learned.FNO(0, seed=0)
n.set_params(d["p"])
z = n.forward(d["chi"], d["k0h"], d["r"])
loss, g = n.loss_grad(d["chi"], d["k0h"], d["r"], d["x"])
np.savez(sys.argv[3], z=z, loss=np.float64(loss), g=g)
"""


def test_fno_tensor_core_dft_matches_cuda_core_path(net, tmp_path, capsys):
    """The same network, inputs and parameters at W = 1024 through the
    tensor-core column DFTs (this process) and through the CUDA-core ones
    (a child process with CUGMRES_FNO_TC_DFT=0): forward output and every
    gradient block agree to the BF16 rounding of the tensor-core path's Z and
    twiddles.  Also records the error of each path against the oracle."""
    import os
    import subprocess
    import sys
    from conftest import ROOT
    p = _params(5)
    chi, k0h, r, x = _inputs(1, 32, 1024, 13)
    net.set_params(p)
    net.set_local_last(True)
    z_tc = net.forward(chi, k0h, r)
    loss_tc, g_tc = net.loss_grad(chi, k0h, r, x)
    inp, out = tmp_path / "in.npz", tmp_path / "out.npz"
    np.savez(inp, p=p, chi=chi, k0h=k0h, r=r, x=x)
    env = dict(os.environ, CUGMRES_FNO_TC_DFT="0")
    res = subprocess.run([sys.executable, "-c", _CUDA_CORE_SCRIPT, ROOT, str(inp), str(out)], env=env,
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    d = np.load(out)
    ref = FO.forward(p, chi, k0h, r, bf16=True)
    sc = ref["s"].numpy().reshape(-1, 1, 1)
    corr_ref = (ref["z"].numpy() - r) / sc

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    e_paths = rel((z_tc - r) / sc, (d["z"] - r) / sc)
    e_tc, e_cc = rel((z_tc - r) / sc, corr_ref), rel((d["z"] - r) / sc, corr_ref)
    assert e_paths < 1e-2, e_paths
    assert abs(loss_tc - float(d["loss"])) <= 5e-3 * abs(float(d["loss"]))
    worst = 0.0
    for a, b in ((FO.OFF_P, FO.OFF_L0), (FO.OFF_L0, FO.OFF_Q1), (FO.OFF_Q1, FO.NPARAM)):
        worst = max(worst, rel(g_tc[a:b], d["g"][a:b]))
    assert worst < 5e-2, worst
    with capsys.disabled():
        print(f"\n  W=1024 correction vs oracle: tensor-core {e_tc:.2e}, CUDA-core {e_cc:.2e}; "
              f"between the paths {e_paths:.2e}; gradients between the paths (worst block) {worst:.2e}")


def test_fno_zero_input_gives_zero(net):
    net.set_params(_params(4))
    chi, k0h, r, _ = _inputs(1, 32, 32, 5)
    z = net.forward(chi, k0h, np.zeros_like(r))
    assert np.all(z == 0)


@pytest.fixture(scope="module")
def trained(cuda_device):
    """A network trained on solver-generated pairs at 48 x 48 (small, for the test's time budget)."""
    data = learned.generate_pairs(48, designs=48, seed=1000, eps_range=(2.0, 6.0), random_per_design=3,
                                  solve_tol=1e-7)
    n = learned.FNO(0, seed=1)
    l0 = learned.evaluate_loss(n, data)
    hist = learned.train(n, data, steps=600, batch=16, lr=2e-3)
    l1 = learned.evaluate_loss(n, data)
    yield n, data, l0, l1, hist
    n.close()


def test_fno_training_reduces_loss(trained):
    _, data, l0, l1, hist = trained
    assert data["unconverged"] == 0
    assert l1 < 0.5 * l0, (l0, l1)


@pytest.fixture(scope="module")
def trained_res(cuda_device):
    """A network trained on the residual loss ||A M(r) - r||^2 / ||r||^2 over the
    solver's own operators (48 x 48 designs)."""
    ds = learned.DesignSet(48, 48, seed=500, eps_range=(2.0, 6.0))
    n = learned.FNO(0, seed=1)
    hist = learned.train_residual(n, ds, steps=1500, batch=16, lr=1e-3)
    ds.close()
    yield n, hist
    n.close()


def test_residual_training_reduces_loss(trained_res):
    hist = trained_res[1]
    assert np.mean(hist[-100:]) < 0.05 * np.mean(hist[:10]), (np.mean(hist[:10]), np.mean(hist[-100:]))


def test_learned_initial_guess_gain_and_fgmres_parity(trained_res, solver, capsys):
    """What the trained network gains: as initial guess, x0 = M(b) starts the
    solve from a fraction of the zero guess's residual on held-out designs.  As
    flexible right preconditioner it gives the same converged solution; its
    iteration ratio against plain GMRES is recorded (at these sizes the
    network does not reduce the iteration count)."""
    n = trained_res[0]
    rows = []
    for seed in (20001, 20002, 20003):
        pr = problems.helmholtz(48, 4.0, seed=seed, cells_per_wavelength=20.0)
        solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
        k0h = pr["k0"] * pr["h"]
        x0 = n.forward(pr["chi"].astype(np.float32), k0h, pr["b"].astype(np.complex64)).astype(np.complex128)
        _, rel0 = solver.residual(pr["b"], x0)
        assert rel0 < 0.8, rel0  # zero initial guess: relative residual 1
        solver.set_preconditioner(n, k0h)
        xa, ia = solver.solve(pr["b"], restart=200, max_iter=2000, tol=1e-10)
        xb, ib = solver.solve(pr["b"], restart=200, max_iter=2000, tol=1e-10, preconditioner="learned",
                              learned_x0=True)
        solver.set_preconditioner(None)
        assert ia["status"] == 0 and ib["status"] == 0
        assert ib["rel_residual_true"] <= 1e-10 and ib["x0_learned"] == 1 and ib["preconditioned_cycles"] >= 1
        assert np.linalg.norm(xb - xa) / np.linalg.norm(xa) < 1e-7
        rows.append((seed, rel0, ia["iterations"], ib["iterations"]))
    with capsys.disabled():
        print("\n  learned x0 residual / plain its / learned its:", rows)


def test_fgmres_fallback_with_bad_network(solver, cuda_device):
    bad = learned.FNO(0, seed=2)
    p = bad.get_params()
    p[FO.OFF_Q2:] *= 1e4  # a network whose corrections are huge and useless
    bad.set_params(p)
    pr = problems.helmholtz(48, 4.0, seed=20004)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    solver.set_preconditioner(bad, pr["k0"] * pr["h"])
    x, info = solver.solve(pr["b"], restart=60, max_iter=3000, tol=1e-10, preconditioner="learned",
                           learned_x0=True)
    solver.set_preconditioner(None)
    bad.close()
    assert info["status"] == 0 and info["rel_residual_true"] <= 1e-10
    assert info["x0_learned"] == 0  # M(b) did not lower the residual and was discarded


def test_fgmres_mixed_precision_learned(trained_res, solver):
    n = trained_res[0]
    pr = problems.helmholtz(48, 4.0, seed=20005)
    solver.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
    solver.set_preconditioner(n, pr["k0"] * pr["h"])
    x, info = solver.solve(pr["b"], restart=100, max_iter=3000, tol=1e-10, precision="mixed",
                           preconditioner="learned", learned_x0=True)
    solver.set_preconditioner(None)
    assert info["status"] == 0 and info["rel_residual_true"] <= 1e-10
