"""CPU oracle of the learned preconditioner (spectral-convolution network).

Test infrastructure only: the parity tests, smoke() and nothing else import
this module; the library never calls it.

The network (no counterpart in the reference; the construction is the
Fourier neural operator of Li et al., ICLR 2021) maps (chi, k0 h, r) to
M(r) = r + s (o0 + i o1), s = rms(r), with

    f   = [0.1 chi, k0 h, Re r / s, Im r / s]
    v0  = P f + p
    z_l = W_l v_l + b_l + S_l(v_l)     S_l(v) = irfft2(trunc(rfft2(v)) * R_l)
    v_l+1 = GELU(z_l) (l < 3), v_4 = z_3
    o   = Q2 GELU(Q1 v_4 + bq1) + bq2

S_l keeps row frequencies 0..15 and H-16..H-1 and column frequencies 0..15
of numpy/torch's real 2-D FFT, mixes channels per mode with a complex
32 x 32 matrix, and applies torch.fft.irfft2 to the truncated spectrum -- an
implementation independent of the library's own truncated-DFT kernels.

`forward(..., bf16=True)` rounds to BF16 exactly where the GPU stores BF16
(activations v_l, pre-activations z_l, the projection's hidden zq, the
tensor-core weights W_l and Q1).  `loss_grad` is a manual backward pass that
follows the GPU's order (including the BF16 rounding of the gradients it
stores); `loss_grad_autograd` is torch autograd of the same loss without any
rounding, which pins the manual formulas.
"""
import numpy as np
import torch

C, NIN, HID, M1, M2, LAYERS = 32, 4, 128, 16, 16, 4
RSZ = 2 * M1 * M2 * C * C * 2
LSZ = RSZ + C * C + C
OFF_P, OFF_PB, OFF_L0 = 0, C * NIN, C * NIN + C
OFF_Q1 = OFF_L0 + LAYERS * LSZ
OFF_BQ1 = OFF_Q1 + HID * C
OFF_Q2 = OFF_BQ1 + HID
OFF_BQ2 = OFF_Q2 + 2 * HID
NPARAM = OFF_BQ2 + 2
CHI_SCALE = 0.1


def off_r(l):
    return OFF_L0 + l * LSZ


def unpack(flat, dtype=torch.float32):
    """Flat parameter vector -> dict of tensors (views in the layout of
    cugmres_fno_get_params)."""
    t = torch.as_tensor(np.asarray(flat, dtype=np.float32)).to(dtype)
    p = {"P": t[OFF_P:OFF_PB].reshape(C, NIN), "pb": t[OFF_PB:OFF_L0]}
    for l in range(LAYERS):
        o = off_r(l)
        p[f"R{l}"] = torch.view_as_complex(t[o:o + RSZ].reshape(2 * M1, M2, C, C, 2).contiguous())
        p[f"W{l}"] = t[o + RSZ:o + RSZ + C * C].reshape(C, C)
        p[f"b{l}"] = t[o + RSZ + C * C:o + LSZ]
    p["Q1"] = t[OFF_Q1:OFF_BQ1].reshape(HID, C)
    p["bq1"] = t[OFF_BQ1:OFF_Q2]
    p["Q2"] = t[OFF_Q2:OFF_BQ2].reshape(2, HID)
    p["bq2"] = t[OFF_BQ2:NPARAM]
    return p


def pack(p):
    """dict of tensors -> flat float32 numpy vector."""
    out = np.zeros(NPARAM, np.float32)
    out[OFF_P:OFF_PB] = p["P"].detach().reshape(-1).float().numpy()
    out[OFF_PB:OFF_L0] = p["pb"].detach().float().numpy()
    for l in range(LAYERS):
        o = off_r(l)
        out[o:o + RSZ] = torch.view_as_real(p[f"R{l}"].detach().to(torch.complex64)).reshape(-1).numpy()
        out[o + RSZ:o + RSZ + C * C] = p[f"W{l}"].detach().reshape(-1).float().numpy()
        out[o + RSZ + C * C:o + LSZ] = p[f"b{l}"].detach().float().numpy()
    out[OFF_Q1:OFF_BQ1] = p["Q1"].detach().reshape(-1).float().numpy()
    out[OFF_BQ1:OFF_Q2] = p["bq1"].detach().float().numpy()
    out[OFF_Q2:OFF_BQ2] = p["Q2"].detach().reshape(-1).float().numpy()
    out[OFF_BQ2:NPARAM] = p["bq2"].detach().float().numpy()
    return out


def _rb(x, on):
    return x.to(torch.bfloat16).to(x.dtype) if on else x


def gelu(x):
    return 0.5 * x * (1.0 + torch.erf(x / np.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1.0 + torch.erf(x / np.sqrt(2.0))) + x * torch.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def spectral(v, R):
    """S(v) for v [B, H, W, C] real, R [32, 16, C, C] complex."""
    B, H, W, _ = v.shape
    vh = torch.fft.rfft2(v.permute(0, 3, 1, 2))  # [B, C, H, W//2+1]
    rows = list(range(M1)) + list(range(H - M1, H))
    xm = vh[:, :, rows, :M2]  # [B, C, 32, 16]
    ym = torch.einsum("bcij,ijco->boij", xm, R)
    full = torch.zeros(B, C, H, W // 2 + 1, dtype=ym.dtype)
    full[:, :, rows, :M2] = ym
    return torch.fft.irfft2(full, s=(H, W)).permute(0, 2, 3, 1)


def features(chi, k0h, r):
    """(f [B,H,W,4], s [B], inv_s [B]) with the GPU's conventions."""
    r = torch.as_tensor(r)
    B = r.shape[0]
    rr = torch.view_as_real(r.to(torch.complex128))
    s = torch.sqrt((rr ** 2).sum(dim=(1, 2, 3)) / (r.shape[1] * r.shape[2]))
    inv_s = torch.where(s > 0, 1.0 / s, torch.ones_like(s)).to(torch.float32)
    s = s.to(torch.float32)
    r32 = torch.view_as_real(r.to(torch.complex64))
    f = torch.stack([torch.as_tensor(chi, dtype=torch.float32) * CHI_SCALE,
                     torch.as_tensor(k0h, dtype=torch.float32).reshape(B, 1, 1).expand(B, r.shape[1], r.shape[2]),
                     r32[..., 0] * inv_s.reshape(B, 1, 1), r32[..., 1] * inv_s.reshape(B, 1, 1)], dim=-1)
    return f, s, inv_s


def forward(flat, chi, k0h, r, bf16=True, keep=False, local_last=True):
    """M(r) (complex64 [B,H,W]), the raw outputs o [B,H,W,2] and, with keep,
    the intermediates of the backward pass.  local_last=False: the last
    Fourier layer has no pointwise path (W_3 is not used)."""
    p = unpack(flat)
    f, s, inv_s = features(chi, k0h, r)
    v = _rb(f @ p["P"].T + p["pb"], bf16)
    acts, zs, X2 = [v], [], []
    for l in range(LAYERS):
        Wl = _rb(p[f"W{l}"], bf16)
        sp = spectral(v, p[f"R{l}"])
        if l == LAYERS - 1 and not local_last:
            Wl = torch.zeros_like(Wl)
        z = v @ Wl.T + p[f"b{l}"] + sp
        zs.append(_rb(z, bf16))
        v = _rb(gelu(z) if l < LAYERS - 1 else z, bf16)
        acts.append(v)
    zq = v @ _rb(p["Q1"], bf16).T + p["bq1"]
    o = gelu(zq) @ p["Q2"].T + p["bq2"]
    rc = torch.as_tensor(r).to(torch.complex64)
    z_out = rc + s.reshape(-1, 1, 1) * torch.complex(o[..., 0], o[..., 1])
    res = {"z": z_out, "o": o, "s": s, "inv_s": inv_s}
    if keep:
        res.update(acts=acts, zs=zs, zq=_rb(zq, bf16), f=f, p=p)
    return res


def _targets(r, x, inv_s):
    r = torch.as_tensor(r).to(torch.complex64)
    x = torch.as_tensor(x).to(torch.complex64)
    t = (x - r) * inv_s.reshape(-1, 1, 1)
    t = torch.view_as_real(t)
    tn = (t.double() ** 2).sum(dim=(1, 2, 3))
    wts = (1.0 / (t.shape[0] * torch.clamp(tn, min=1e-30))).float()
    return t, wts


def loss_grad(flat, chi, k0h, r, x, bf16=True, local_last=True):
    """(loss, grad flat float32) by the manual backward pass of the GPU."""
    fw = forward(flat, chi, k0h, r, bf16=bf16, keep=True, local_last=local_last)
    p, o, inv_s = fw["p"], fw["o"], fw["inv_s"]
    t, wts = _targets(r, x, inv_s)
    w = wts.reshape(-1, 1, 1, 1)
    d = o - t
    loss = float((w.double() * d.double() ** 2).sum())
    dout = 2.0 * w * d
    g = {}
    zq = fw["zq"]  # rounded as stored
    g["Q2"] = torch.einsum("bhwk,bhwj->kj", dout, gelu(zq))
    g["bq2"] = dout.sum(dim=(0, 1, 2))
    dzq = _rb((dout @ p["Q2"]) * gelu_d(zq), bf16)
    v4 = fw["acts"][LAYERS]
    g["Q1"] = torch.einsum("bhwj,bhwc->jc", dzq, v4)
    g["bq1"] = dzq.sum(dim=(0, 1, 2))
    dz = _rb(dzq @ _rb(p["Q1"], bf16), bf16)
    for l in range(LAYERS - 1, -1, -1):
        vl = fw["acts"][l]
        g[f"W{l}"] = torch.einsum("bhwo,bhwc->oc", dz, vl)
        g[f"b{l}"] = dz.sum(dim=(0, 1, 2))
        # adjoint of the (linear) spectral branch by autograd: d/dv and d/dR at the cotangent dz
        vv = vl.clone().requires_grad_(True)
        RR = p[f"R{l}"].clone().requires_grad_(True)
        out = spectral(vv, RR)
        gv, gR = torch.autograd.grad(out, (vv, RR), grad_outputs=dz)
        g[f"R{l}"] = gR  # torch's gradient of a real loss w.r.t. a complex leaf is d/dRe + i d/dIm
        if l == LAYERS - 1 and not local_last:
            g[f"W{l}"] = torch.zeros_like(g[f"W{l}"])
            dv = gv
        else:
            dv = dz @ _rb(p[f"W{l}"], bf16) + gv
        if l > 0:
            dz = _rb(dv * gelu_d(fw["zs"][l - 1]), bf16)
        else:
            dv0 = dv
    g["P"] = torch.einsum("bhwc,bhwj->cj", dv0, fw["f"])
    g["pb"] = dv0.sum(dim=(0, 1, 2))
    return loss, pack(g)


def loss_grad_autograd(flat, chi, k0h, r, x, dtype=torch.float64, local_last=True):
    """(loss, grad) of the same loss by torch autograd, without BF16 rounding."""
    p = {k: v.to(dtype if not v.is_complex() else torch.complex128).clone().requires_grad_(True)
         for k, v in unpack(flat).items()}
    f, s, inv_s = features(chi, k0h, r)
    f = f.to(dtype)
    v = f @ p["P"].T + p["pb"]
    for l in range(LAYERS):
        Wl = p[f"W{l}"] if (l < LAYERS - 1 or local_last) else 0.0 * p[f"W{l}"]
        z = v @ Wl.T + p[f"b{l}"] + spectral(v, p[f"R{l}"])
        v = gelu(z) if l < LAYERS - 1 else z
    o = gelu(v @ p["Q1"].T + p["bq1"]) @ p["Q2"].T + p["bq2"]
    t, wts = _targets(r, x, inv_s)
    loss = (wts.to(dtype).reshape(-1, 1, 1, 1) * (o - t.to(dtype)) ** 2).sum()
    loss.backward()
    g = {k: v.grad for k, v in p.items()}
    return float(loss.detach()), pack(g)
