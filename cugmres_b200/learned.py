"""Learned preconditioner: a spectral-convolution network trained on solutions
the solver itself generates, used as initial guess and as the variable right
preconditioner of flexible GMRES (cugmres_fno_* and cugmres_set_preconditioner
of the C-ABI; inference and training kernels are the library's own CUDA).

    net = FNO(device=0, seed=0)
    data = generate_pairs(64, designs=256, seed=1000)      # solver-generated (r, x) pairs
    train(net, data, steps=2000)
    solver.set_preconditioner(net, k0h)
    x, info = solver.solve(b, preconditioner="learned")

The network sees r normalised by its RMS, so M(a r) = a M(r) for a > 0.
"""
import ctypes
import time

import numpy as np

from . import _lib
from ._lib import check


def _carr(a, dtype):
    """(c_void_p, keepalive) for a NumPy array or a contiguous CUDA torch tensor of `dtype`."""
    if type(a).__module__.split(".")[0] == "torch":
        if not a.is_contiguous():
            raise TypeError("tensor must be contiguous")
        return ctypes.c_void_p(a.data_ptr()), a
    arr = np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data_as(ctypes.c_void_p), arr


class FNO:
    """The network on one GPU (parameters, optimiser state and workspace)."""

    def __init__(self, device=0, seed=0):
        self._net = ctypes.c_void_p()
        check(_lib.lib().cugmres_fno_create(ctypes.byref(self._net), int(device), int(seed)), "fno_create")
        self.device = int(device)

    def close(self):
        if self._net:
            _lib.lib().cugmres_fno_destroy(self._net)
            self._net = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_local_last(self, on):
        """False: the last Fourier layer is spectral only (band-limited correction)."""
        check(_lib.lib().cugmres_fno_set_local_last(self._net, int(bool(on))), "fno_set_local_last")

    def info(self):
        i = _lib.CgFnoInfo()
        check(_lib.lib().cugmres_fno_info(self._net, ctypes.byref(i)), "fno_info")
        return {k: getattr(i, k) for k, _ in i._fields_}

    @property
    def num_params(self):
        return self.info()["num_params"]

    def get_params(self):
        out = np.empty(self.num_params, np.float32)
        check(_lib.lib().cugmres_fno_get_params(self._net, out.ctypes.data_as(ctypes.c_void_p)), "fno_get_params")
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {p.size}")
        check(_lib.lib().cugmres_fno_set_params(self._net, p.ctypes.data_as(ctypes.c_void_p)), "fno_set_params")

    @staticmethod
    def _batch(chi, k0h, r):
        r = np.asarray(r) if not type(r).__module__.startswith("torch") else r
        if r.ndim == 2:
            r = r[None]
            chi = np.asarray(chi)[None]
        B, H, W = r.shape
        k0h = np.broadcast_to(np.asarray(k0h, np.float32).reshape(-1), (B,)).copy()
        return B, H, W, chi, k0h, r

    def forward(self, chi, k0h, r):
        """M(r) (complex64, same shape as r) for r [B, H, W] or [H, W]."""
        squeeze = np.ndim(r) == 2
        B, H, W, chi, k0h, r = self._batch(chi, k0h, r)
        cp, ck = _carr(chi, np.float32)
        kp, kk = _carr(k0h, np.float32)
        rp, rk = _carr(r, np.complex64)
        z = np.empty((B, H, W), np.complex64)
        check(_lib.lib().cugmres_fno_forward(self._net, B, H, W, cp, kp, rp, z.ctypes.data_as(ctypes.c_void_p)),
              "fno_forward")
        return z[0] if squeeze else z

    def loss_grad(self, chi, k0h, r, x):
        B, H, W, chi, k0h, r = self._batch(chi, k0h, r)
        x = np.asarray(x)[None] if np.ndim(x) == 2 else x
        cp, ck = _carr(chi, np.float32)
        kp, kk = _carr(k0h, np.float32)
        rp, rk = _carr(r, np.complex64)
        xp, xk = _carr(x, np.complex64)
        loss = ctypes.c_float(0.0)
        g = np.empty(self.num_params, np.float32)
        check(_lib.lib().cugmres_fno_loss_grad(self._net, B, H, W, cp, kp, rp, xp, ctypes.byref(loss),
                                               g.ctypes.data_as(ctypes.c_void_p)), "fno_loss_grad")
        return loss.value, g

    def train_step(self, chi, k0h, r, x, lr):
        B, H, W, chi, k0h, r = self._batch(chi, k0h, r)
        cp, ck = _carr(chi, np.float32)
        kp, kk = _carr(k0h, np.float32)
        rp, rk = _carr(r, np.complex64)
        xp, xk = _carr(x, np.complex64)
        loss = ctypes.c_float(0.0)
        check(_lib.lib().cugmres_fno_train_step(self._net, B, H, W, cp, kp, rp, xp, float(lr), ctypes.byref(loss)),
              "fno_train_step")
        return loss.value

    def forward_train(self, chi, k0h, r):
        """M(r) for a batch, keeping what backward() needs."""
        B, H, W, chi, k0h, r = self._batch(chi, k0h, r)
        cp, ck = _carr(chi, np.float32)
        kp, kk = _carr(k0h, np.float32)
        rp, rk = _carr(r, np.complex64)
        z = np.empty((B, H, W), np.complex64)
        check(_lib.lib().cugmres_fno_forward_train(self._net, B, H, W, cp, kp, rp,
                                                   z.ctypes.data_as(ctypes.c_void_p)), "fno_forward_train")
        return z

    def backward(self, dm, lr=0.0, want_grad=False):
        """Backward pass from dL/dM (complex, d/dRe + i d/dIm) of the last
        forward_train batch; Adam step when lr > 0.  Returns the gradient if asked."""
        d = np.ascontiguousarray(dm, np.complex64)
        g = np.empty(self.num_params, np.float32) if want_grad else None
        check(_lib.lib().cugmres_fno_backward(self._net, d.ctypes.data_as(ctypes.c_void_p),
                                              g.ctypes.data_as(ctypes.c_void_p) if want_grad else None,
                                              float(lr)), "fno_backward")
        return g

    def save(self, path, **meta):
        np.savez_compressed(path, params=self.get_params(), **{k: np.asarray(v) for k, v in meta.items()})

    def load(self, path):
        with np.load(path) as d:
            self.set_params(d["params"])


# ------------------------------------------------------------------ data
def smooth_field(N, rng, corr):
    """Complex Gaussian random field with correlation length `corr` cells (periodic, unit RMS)."""
    w = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    f = np.fft.fftfreq(N)
    filt = np.exp(-2.0 * (np.pi * corr) ** 2 * (f[:, None] ** 2 + f[None, :] ** 2))
    v = np.fft.ifft2(np.fft.fft2(w) * filt)
    return v / np.sqrt(np.mean(np.abs(v) ** 2))


def generate_pairs(N, designs, seed, eps_range=(2.0, 12.0), lh_range=(15.0, 30.0), random_per_design=3,
                   solve_tol=1e-7, max_iter=3000, device=0, solver=None, log=None):
    """Training pairs (chi, k0h, r, x) with A x = r, all produced by this
    library's solver on seeded random designs (the thresholded Gaussian-field
    contrast of problems.helmholtz, eps_r ~ U(eps_range), lambda/h ~ U(lh_range)):

    * one plane-wave right-hand side per design at a random incidence angle,
      solved to `solve_tol` by GMRES (the initial-guess use);
    * `random_per_design` smooth random fields y (correlation 1..8 cells),
      r = A y computed by the solver's FFT matvec, x = y (the preconditioner
      use: M is applied to arbitrary Krylov vectors).
    """
    from . import Solver
    from . import problems
    rng = np.random.default_rng(seed)
    own = solver is None
    s = Solver(device) if own else solver
    chis, k0hs, rs, xs = [], [], [], []
    t0 = time.time()
    unconverged = 0
    for d in range(designs):
        eps = float(rng.uniform(*eps_range))
        lh = float(rng.uniform(*lh_range))
        pr = problems.helmholtz(N, eps, seed=int(rng.integers(1 << 30)), cells_per_wavelength=lh)
        s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
        k0h = pr["k0"] * pr["h"]
        th = rng.uniform(0, 2 * np.pi)
        xc = (np.arange(N) + 0.5) * pr["h"]
        b = np.exp(1j * pr["k0"] * (np.cos(th) * xc[:, None] + np.sin(th) * xc[None, :]))
        x, info = s.solve(b, restart=max(50, min(max_iter, 200)), max_iter=max_iter, tol=solve_tol)
        if info["status"] != 0:
            unconverged += 1
        chis.append(pr["chi"].astype(np.float32))
        k0hs.append(k0h)
        rs.append(b.astype(np.complex64))
        xs.append(x.astype(np.complex64))
        for _ in range(random_per_design):
            y = smooth_field(N, rng, rng.uniform(1.0, 8.0))
            chis.append(pr["chi"].astype(np.float32))
            k0hs.append(k0h)
            rs.append(s.matvec(y).astype(np.complex64))
            xs.append(y.astype(np.complex64))
        if log and (d + 1) % max(1, designs // 8) == 0:
            log(f"  pairs: {d + 1}/{designs} designs, {time.time() - t0:.1f} s")
    if own:
        s.close()
    return dict(N=N, chi=np.stack(chis), k0h=np.asarray(k0hs, np.float32), r=np.stack(rs), x=np.stack(xs),
                unconverged=unconverged, seconds=time.time() - t0)


class DesignSet:
    """Seeded random designs with one solver context each (operators set once),
    for training on the residual-space loss."""

    def __init__(self, N, count, seed, eps_range=(2.0, 12.0), lh_range=(15.0, 30.0), device=0, krylov=12):
        from . import Solver
        from . import problems
        rng = np.random.default_rng(seed)
        self.N = N
        self.items = []
        for _ in range(count):
            eps = float(rng.uniform(*eps_range))
            lh = float(rng.uniform(*lh_range))
            pr = problems.helmholtz(N, eps, seed=int(rng.integers(1 << 30)), cells_per_wavelength=lh)
            s = Solver(device)
            s.set_operator(pr["g_block"], pr["chi"], pr["chi_scale"])
            th = rng.uniform(0, 2 * np.pi)
            xc = (np.arange(N) + 0.5) * pr["h"]
            b = np.exp(1j * pr["k0"] * (np.cos(th) * xc[:, None] + np.sin(th) * xc[None, :]))
            kv = [b / np.linalg.norm(b)]  # Krylov sequence A^j b (normalised)
            for _ in range(krylov):
                v = s.matvec(kv[-1])
                kv.append(v / np.linalg.norm(v))
            self.items.append(dict(solver=s, chi=pr["chi"].astype(np.float32), k0h=pr["k0"] * pr["h"], b=b,
                                   krylov=np.stack(kv), eps=eps, lh=lh, k0=pr["k0"], h=pr["h"]))

    def close(self):
        for it in self.items:
            it["solver"].close()
        self.items = []

    def A(self, i, z):
        return self.items[i]["solver"].matvec(np.ascontiguousarray(z, np.complex128))

    def AH(self, i, e):
        """A^H e = conj(A^T conj(e))."""
        return np.conj(self.items[i]["solver"].matvec(np.ascontiguousarray(np.conj(e), np.complex128),
                                                      transpose=True))

    def sample_input(self, i, rng):
        """A right-hand side of the kinds M meets: Krylov vectors, plane waves, smooth and white fields."""
        it, N = self.items[i], self.N
        u = rng.random()
        if u < 0.4:
            return it["krylov"][rng.integers(len(it["krylov"]))]
        if u < 0.55:
            return it["b"]
        if u < 0.85:
            return smooth_field(N, rng, rng.uniform(0.5, 8.0))
        w = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
        return w / np.sqrt(2.0)


def train_residual(net, designs, steps=1000, batch=16, lr=1e-3, lr_min=1e-5, seed=0, log=None, log_every=100):
    """Adam on the preconditioning loss (1/B) sum ||A M(r) - r||^2 / ||r||^2 over
    inputs drawn by DesignSet.sample_input; dL/dM = 2 A^H (A M(r) - r) / (B ||r||^2)."""
    rng = np.random.default_rng(seed)
    n = len(designs.items)
    hist = []
    t0 = time.time()
    for it in range(steps):
        idx = rng.integers(0, n, size=batch)
        r = np.stack([designs.sample_input(i, rng) for i in idx]).astype(np.complex64)
        chi = np.stack([designs.items[i]["chi"] for i in idx])
        k0h = np.asarray([designs.items[i]["k0h"] for i in idx], np.float32)
        z = net.forward_train(chi, k0h, r)
        dm = np.empty_like(z)
        loss = 0.0
        for q, i in enumerate(idx):
            rr = r[q].astype(np.complex128)
            e = designs.A(i, z[q].astype(np.complex128)) - rr
            nr = np.vdot(rr, rr).real
            loss += np.vdot(e, e).real / nr / batch
            dm[q] = (2.0 / (batch * nr)) * designs.AH(i, e)
        a = lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * it / max(1, steps)))
        net.backward(dm, lr=a)
        hist.append(loss)
        if log and (it % log_every == 0 or it == steps - 1):
            log(f"  step {it:5d}  residual loss {np.mean(hist[-log_every:]):.4f}  lr {a:.2e}  {time.time() - t0:.1f} s")
    return np.asarray(hist)


def train(net, data, steps=2000, batch=16, lr=1e-3, lr_min=1e-5, seed=0, log=None, log_every=200):
    """Adam with cosine learning-rate decay over random mini-batches of `data`."""
    rng = np.random.default_rng(seed)
    n = data["r"].shape[0]
    hist = []
    t0 = time.time()
    for it in range(steps):
        idx = rng.choice(n, size=min(batch, n), replace=False)
        a = lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * it / max(1, steps)))
        loss = net.train_step(data["chi"][idx], data["k0h"][idx], data["r"][idx], data["x"][idx], a)
        hist.append(loss)
        if log and (it % log_every == 0 or it == steps - 1):
            log(f"  step {it:5d}  loss {np.mean(hist[-log_every:]):.4f}  lr {a:.2e}  {time.time() - t0:.1f} s")
    return np.asarray(hist)


def evaluate_loss(net, data, batch=16):
    """Mean loss over `data` (relative squared error of the correction)."""
    n = data["r"].shape[0]
    tot, cnt = 0.0, 0
    for i in range(0, n, batch):
        sl = slice(i, min(n, i + batch))
        l, _ = net.loss_grad(data["chi"][sl], data["k0h"][sl], data["r"][sl], data["x"][sl])
        tot += l * (sl.stop - sl.start)
        cnt += sl.stop - sl.start
    return tot / max(1, cnt)
