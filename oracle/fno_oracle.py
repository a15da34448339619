"""CPU FP32 oracle of the surrogate network (test infrastructure only).

The same Fourier neural operator as seisfem_b200/surrogate.py, written with
torch on the CPU in FP32 and differentiated by autograd.  The spectral
convolution uses torch.fft (rfft2 / irfft2 with the kept modes 0..15 and
D-16..D-1 along depth, 0..15 along the receiver axis, as in the standard FNO
formulation), which checks the GPU's explicit DFT-matrix GEMMs independently.
Parameters are the dict of float32 arrays ``init_params`` returns.
"""
from __future__ import annotations

import numpy as np
import torch

KC = 16


def _spectral(v, wr, wi):
    # v [B][C][D][W]; wr, wi [32*16][C][C] (mode = k1 * 16 + k2, k1 over 0..15, D-16..D-1)
    B, Cc, D, W = v.shape
    vf = torch.fft.rfft2(v)                            # [B][C][D][W/2+1]
    w = torch.complex(wr, wi).reshape(2, KC, KC, Cc, Cc)   # [half][k1][k2][i][o]
    out = torch.zeros(B, Cc, D, W // 2 + 1, dtype=torch.complex64)
    lo = vf[:, :, :KC, :KC]
    hi = vf[:, :, D - KC:, :KC]
    out[:, :, :KC, :KC] = torch.einsum("bixy,xyio->boxy", lo, w[0])
    out[:, :, D - KC:, :KC] = torch.einsum("bixy,xyio->boxy", hi, w[1])
    return torch.fft.irfft2(out, s=(D, W))


def forward(params: dict, x: np.ndarray, layers: int = 4):
    """x [B][cin][D][W] -> (y [B][2][W][T], tensors with requires_grad)."""
    P = {k: torch.tensor(v, dtype=torch.float32, requires_grad=True) for k, v in params.items()}
    xt = torch.tensor(x, dtype=torch.float32)
    B, cin, D, W = xt.shape
    v = torch.einsum("ci,bidw->bcdw", P["lift_w"], xt) + P["lift_b"][None, :, None, None]
    for l in range(layers):
        s = _spectral(v, P[f"wr{l}"], P[f"wi{l}"])
        pre = s + torch.einsum("oi,bidw->bodw", P[f"cw{l}"], v) + P[f"cb{l}"][None, :, None, None]
        v = torch.nn.functional.gelu(pre) if l < layers - 1 else pre
    u = torch.einsum("bcdw,dt->bcwt", v, P["time_w"]) + P["time_b"]
    h = torch.nn.functional.gelu(torch.einsum("bcwt,cj->bwtj", u, P["p1_w"]) + P["p1_b"])
    y = torch.einsum("bwtj,jk->bkwt", h, P["p2_w"]) + P["p2_b"][None, :, None, None]
    return y, P


def loss_and_grads(params: dict, x: np.ndarray, target: np.ndarray, layers: int = 4):
    """Mean over shots of |y - target|^2 / |target|^2 and its gradients."""
    y, P = forward(params, x, layers)
    t = torch.tensor(target, dtype=torch.float32)
    B = y.shape[0]
    num = ((y - t) ** 2).reshape(B, -1).sum(1)
    den = (t ** 2).reshape(B, -1).sum(1)
    loss = (num / den).mean()
    loss.backward()
    return y.detach().numpy(), (num / den).detach().numpy(), {k: v.grad.numpy() for k, v in P.items()}
