"""CPU emulation of the sfg_fno_* kernels (test infrastructure).

Implements each entry point with torch on the CPU, with the same strided
operand addressing (torch.as_strided over the flat buffers, element offsets
and strides exactly as the GEMM descriptor gives them) and the same BF16
rounding points, so the surrogate's host sequencing -- every stride, offset
and buffer layout of seisfem_b200/surrogate.py -- can be checked on a
machine without a GPU against the FP32 oracle (oracle/fno_oracle.py)."""
from __future__ import annotations

import torch

KC, KD = 16, 32


def _view(t, size, stride, off):
    # element offsets count from the tensor's first element (which need not
    # start its storage: the gradients are views into one flat buffer)
    return torch.as_strided(t.view(-1), size, stride, t.storage_offset() + off)


class EmuKernels:
    def __init__(self):
        self.launches = 0

    def gemm(self, A, B, Cout, M, N, K, a=(0, 0, 0, 0), b=(0, 0, 0, 0), c=(0, 0, 0, 0), batch=(1, 1),
             aoff=0, boff=0, coff=0, Cin=None, pre=None, bias=None, bias_on_m=False, gelu=False,
             alpha=1.0, beta=1.0, atomic=False, splits=1):
        self.launches += 1
        b1, b2 = batch
        Av = _view(A, (b1, b2, M, K), a, aoff).float()
        Bv = _view(B, (b1, b2, K, N), b, boff).float()
        acc = alpha * torch.matmul(Av, Bv)
        Cv = _view(Cout, (b1, b2, M, N), c, coff)
        if atomic:
            for i in range(b1):
                for j in range(b2):
                    Cv[i, j] += acc[i, j]
            return
        v = acc
        if Cin is not None:
            v = v + beta * _view(Cin, (b1, b2, M, N), c, coff).float()
        if bias is not None:
            v = v + (bias[:M, None] if bias_on_m else bias[None, :N])
        if pre is not None:
            _view(pre, (b1, b2, M, N), c, coff).copy_(v.to(pre.dtype))
        if gelu:
            v = torch.nn.functional.gelu(v)
        Cv.copy_(v.to(Cout.dtype))

    def call(self, name, *args):
        self.launches += 1
        getattr(self, name[len("sfg_fno_"):])(*args)

    # pointwise entry points, argument order of include/seisfem_fno.h
    def dft_combine(self, P, Z, B, C):
        p = P.view(B * C, 64, 32)
        re = p[:, :KD, :KC] + p[:, KD:, KC:]
        im = p[:, :KD, KC:] - p[:, KD:, :KC]
        z = Z.view(KD, KC, B, 2, C)
        z[:, :, :, 0, :] = re.reshape(B, C, KD, KC).permute(2, 3, 0, 1).to(Z.dtype)
        z[:, :, :, 1, :] = im.reshape(B, C, KD, KC).permute(2, 3, 0, 1).to(Z.dtype)

    def dft_combine_bwd(self, dZ, dP, B, C):
        z = dZ.view(KD, KC, B, 2, C)
        re = z[:, :, :, 0, :].permute(2, 3, 0, 1).reshape(B * C, KD, KC)
        im = z[:, :, :, 1, :].permute(2, 3, 0, 1).reshape(B * C, KD, KC)
        p = dP.view(B * C, 64, 32)
        p[:, :KD, :KC] = re
        p[:, KD:, KC:] = re
        p[:, :KD, KC:] = im
        p[:, KD:, :KC] = -im

    def expand_weights(self, Wr, Wi, Wb, modes, C):
        w = Wb.view(modes, 2 * C, 2 * C)
        w[:, :C, :C] = Wr.to(Wb.dtype)
        w[:, :C, C:] = Wi.to(Wb.dtype)
        w[:, C:, :C] = (-Wi).to(Wb.dtype)
        w[:, C:, C:] = Wr.to(Wb.dtype)

    def fold_weights(self, dWb, dWr, dWi, modes, C):
        w = dWb.view(modes, 2 * C, 2 * C)
        dWr += w[:, :C, :C] + w[:, C:, C:]
        dWi += w[:, :C, C:] - w[:, C:, :C]

    def gelu_bwd(self, dy, dy_bf16, pre, dx, n):
        x = pre.view(-1)[:n].float()
        g = dy.view(-1)[:n].float()
        cdf = 0.5 * (1 + torch.erf(x / 2 ** 0.5))
        pdf = torch.exp(-0.5 * x * x) / (2 * torch.pi) ** 0.5
        dx.view(-1)[:n] = (g * (cdf + x * pdf)).to(dx.dtype)

    def cast_bf16(self, x, y, n):
        y.view(-1)[:n] = x.view(-1)[:n].to(y.dtype)

    def bias_grad(self, dy, db, outer, C, inner):
        db += dy.view(outer, C, inner).float().sum(dim=(0, 2))

    def swap01(self, x, y, n0, n1, n2):
        y.view(n1, n0, n2).copy_(x.view(n0, n1, n2).transpose(0, 1))

    def zero(self, p, n):
        p.view(-1)[:n] = 0

    def scale(self, p, n, a):
        p.view(-1)[:n] *= a

    def rel_loss(self, pred, target, loss, dpred, scratch, B, n):
        p = pred.view(B, n)
        t = target.view(B, n).float()
        num = ((p - t) ** 2).sum(1)
        den = (t ** 2).sum(1).clamp_min(1e-30)
        loss[:B] = num / den
        if dpred is not None:
            dpred.view(B, n).copy_((2 * (p - t) / (B * den[:, None])).to(dpred.dtype))

    def adam(self, p, g, m, v, n, lr, b1, b2, eps, step):
        m.mul_(b1).add_((1 - b1) * g)
        v.mul_(b2).add_((1 - b2) * g * g)
        p -= lr * (m / (1 - b1 ** step)) / (torch.sqrt(v / (1 - b2 ** step)) + eps)
