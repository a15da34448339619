"""Learned surrogate: a Fourier neural operator (FNO) that maps a velocity
model and a source position to the receiver gather the FEM records.

No counterpart in the reference.  The FEM of this package generates the
training shots and stays the fallback and judge of the surrogate's error.
Every arithmetic step of the network -- forward, backward and the Adam
update -- runs in this library's own CUDA kernels (``sfg_fno_*`` in
``include/seisfem_fno.h``): a strided batched BF16 tensor-core GEMM with FP32
accumulation plus a few pointwise kernels.  PyTorch only allocates the device
buffers this module hands to those kernels.

Network (width C, 4 Fourier layers, 16 modes per axis):

* input  x[B][4][D][W]: normalised vp, a source-position channel (a Gaussian
  in the horizontal coordinate), depth and horizontal coordinates, on a
  depth x receiver-column grid;
* lift   v0 = Wl x + bl (1x1);
* layer  v_{l+1} = GELU(S_l(v_l) + W_l v_l + b_l) (no GELU after the last),
  S_l the spectral convolution: truncated real DFT along W (16 modes), DFT
  along D (modes 0..15 and D-16..D-1), complex channel mixing per mode,
  inverse transforms -- each a GEMM with fixed DFT matrices;
* time   u[b][c][w][t] = sum_d v4[b][c][d][w] Wt[d][t] + bt[t] (depth to time);
* head   y[b][ch][w][t] = P2 GELU(P1 u + p1) + p2 (per point, 2 channels:
  the u and w displacement gathers).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import api

KC, KD = 16, 32          # kept modes along W and along D (16 + 16)


class GemmDesc(C.Structure):
    _fields_ = [("A", C.c_void_p), ("B", C.c_void_p), ("C", C.c_void_p), ("Cin", C.c_void_p),
                ("pre", C.c_void_p), ("bias", C.c_void_p),
                ("sa1", C.c_longlong), ("sa2", C.c_longlong), ("sam", C.c_longlong), ("sak", C.c_longlong),
                ("sb1", C.c_longlong), ("sb2", C.c_longlong), ("sbk", C.c_longlong), ("sbn", C.c_longlong),
                ("sc1", C.c_longlong), ("sc2", C.c_longlong), ("scm", C.c_longlong), ("scn", C.c_longlong),
                ("M", C.c_int), ("N", C.c_int), ("K", C.c_int), ("batch1", C.c_int), ("batch2", C.c_int),
                ("splits", C.c_int), ("alpha", C.c_float), ("beta", C.c_float),
                ("c_bf16", C.c_int), ("gelu", C.c_int), ("bias_on_m", C.c_int), ("atomic", C.c_int),
                ("engine", C.c_int)]


def _ptr(t, off=0):
    return None if t is None else t.data_ptr() + off * t.element_size()


class Kernels:
    """ctypes front of the sfg_fno_* entry points on one stream."""

    def __init__(self, stream=None):
        self.L = api.lib()
        self.stream = stream
        self.launches = 0
        self.flops = 0          # 2 M N K per problem of every GEMM issued
        # GEMM engine: 0 automatic (tcgen05 for M >= 64, N >= 32, K >= 64), 1 mma.sync,
        # 2 tcgen05 (persistent, TMA operand tiles where the strides allow), 3 tcgen05 with
        # cp.async tiles, 4 tcgen05 with TMA tiles and one output tile per CTA
        self.engine = 0
        f = self.L.sfg_fno_gemm
        f.argtypes = [C.POINTER(GemmDesc), C.c_void_p]
        for n, a in [("sfg_fno_dft_combine", [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
                     ("sfg_fno_dft_combine_bwd", [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
                     ("sfg_fno_expand_weights", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
                     ("sfg_fno_fold_weights", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
                     ("sfg_fno_gelu_bwd", [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p]),
                     ("sfg_fno_cast_bf16", [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p]),
                     ("sfg_fno_bias_grad", [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_longlong, C.c_void_p]),
                     ("sfg_fno_rel_loss", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                           C.c_longlong, C.c_void_p]),
                     ("sfg_fno_adam", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_float,
                                       C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]),
                     ("sfg_fno_swap01", [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_longlong, C.c_void_p]),
                     ("sfg_fno_zero", [C.c_void_p, C.c_longlong, C.c_void_p]),
                     ("sfg_fno_scale", [C.c_void_p, C.c_longlong, C.c_float, C.c_void_p])]:
            getattr(self.L, n).argtypes = a
            getattr(self.L, n).restype = C.c_int
        f.restype = C.c_int

    def _check(self, rc, what):
        self.launches += 1
        if rc:
            raise api.SfgError(rc, what)

    def gemm(self, A, B, Cout, M, N, K, a=(0, 0, 0, 0), b=(0, 0, 0, 0), c=(0, 0, 0, 0), batch=(1, 1),
             aoff=0, boff=0, coff=0, Cin=None, pre=None, bias=None, bias_on_m=False, gelu=False,
             alpha=1.0, beta=1.0, atomic=False, splits=1, engine=None):
        """Strides are (level-1 batch, level-2 batch, row, col) in elements;
        engine 0 automatic, 1 mma.sync, 2 tcgen05 (persistent, TMA tiles), 3 tcgen05 (cp.async
        tiles), 4 tcgen05 (TMA tiles, one output tile per CTA);
        default: self.engine."""
        d = GemmDesc()
        d.A, d.B, d.C = _ptr(A, aoff), _ptr(B, boff), _ptr(Cout, coff)
        d.Cin = _ptr(Cin, coff) if Cin is not None else None
        d.pre = _ptr(pre, coff) if pre is not None else None
        d.bias = _ptr(bias)
        d.sa1, d.sa2, d.sam, d.sak = a
        d.sb1, d.sb2, d.sbk, d.sbn = b
        d.sc1, d.sc2, d.scm, d.scn = c
        d.M, d.N, d.K = M, N, K
        d.batch1, d.batch2, d.splits = batch[0], batch[1], splits
        d.alpha, d.beta = alpha, beta
        import torch
        d.c_bf16 = int(Cout.dtype == torch.bfloat16)
        d.gelu, d.bias_on_m, d.atomic = int(gelu), int(bias_on_m), int(atomic)
        d.engine = self.engine if engine is None else engine
        self.flops += 2 * M * N * K * batch[0] * batch[1]
        self._check(self.L.sfg_fno_gemm(C.byref(d), self.stream), "sfg_fno_gemm")

    def head_infer(self, A, B, y, M, N, K, a, b, batch, bias, w2, b2, y_batch, y_ch):
        """sfg_fno_head_infer: GELU(A B + bias) times w2 (+ b2) into y without
        storing the hidden layer; False when the layout does not fit (the
        caller then runs the two GEMMs)."""
        d = GemmDesc()
        d.A, d.B = _ptr(A), _ptr(B)
        d.bias = _ptr(bias)
        d.sa1, d.sa2, d.sam, d.sak = a
        d.sb1, d.sb2, d.sbk, d.sbn = b
        d.M, d.N, d.K = M, N, K
        d.batch1, d.batch2, d.splits = batch, 1, 1
        d.alpha, d.beta = 1.0, 0.0
        d.gelu = 1
        f = self.L.sfg_fno_head_infer
        f.argtypes = [C.POINTER(GemmDesc), C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_longlong, C.c_int,
                      C.c_void_p]
        f.restype = C.c_int
        rc = f(C.byref(d), _ptr(w2), _ptr(b2), _ptr(y), y_batch, y_ch, w2.shape[1], self.stream)
        if rc == 3:
            return False
        self._check(rc, "sfg_fno_head_infer")
        self.flops += 2 * M * N * K * batch + 2 * M * N * w2.shape[1] * batch
        return True

    def call(self, name, *args):
        """Pointwise entry point `name`; tensor arguments pass as device pointers."""
        import torch
        conv = [a.data_ptr() if isinstance(a, torch.Tensor) else a for a in args]
        self._check(getattr(self.L, name)(*conv, self.stream), name)


def dft_mats(D: int, W: int):
    """The fixed DFT matrices of the spectral convolution (float64):
    Fw[W][32] (rfft along W: cos | -sin), Gd[64][D] (cos rows | sin rows of
    the kept D modes), Gi2[2D][64] (inverse along D, real and imaginary output
    halves), Gw[32][W] (irfft along W, 1/W and 2/W weights)."""
    k1 = np.concatenate([np.arange(KC), np.arange(D - KC, D)])
    w = np.arange(W)
    th = 2 * np.pi * np.outer(w, np.arange(KC)) / W
    Fw = np.concatenate([np.cos(th), -np.sin(th)], axis=1)
    d = np.arange(D)
    ph = 2 * np.pi * np.outer(k1, d) / D            # [32][D]
    Gd = np.concatenate([np.cos(ph), np.sin(ph)], axis=0)
    Gi2 = np.zeros((2 * D, 2 * KD))
    Gi2[:D, :KD] = np.cos(ph).T / D
    Gi2[:D, KD:] = -np.sin(ph).T / D
    Gi2[D:, :KD] = np.sin(ph).T / D
    Gi2[D:, KD:] = np.cos(ph).T / D
    ck = np.full(KC, 2.0 / W)
    ck[0] = 1.0 / W
    Gw = np.concatenate([ck[:, None] * np.cos(th.T), -ck[:, None] * np.sin(th.T)], axis=0)
    return tuple(np.ascontiguousarray(m) for m in (Fw, Gd, Gi2, Gw))


def init_params(C_: int, D: int, T: int, Hp: int, cin: int = 4, layers: int = 4, seed: int = 0):
    """Seeded initial weights (float32 numpy), the layout both this module and
    the CPU oracle use."""
    rng = np.random.default_rng(seed)
    modes = KD * KC
    p = {"lift_w": rng.standard_normal((C_, cin)) / math.sqrt(cin), "lift_b": np.zeros(C_)}
    sc = 1.0 / (C_ * C_)
    for l in range(layers):
        p[f"wr{l}"] = sc * rng.random((modes, C_, C_))
        p[f"wi{l}"] = sc * rng.random((modes, C_, C_))
        p[f"cw{l}"] = rng.standard_normal((C_, C_)) / math.sqrt(C_)
        p[f"cb{l}"] = np.zeros(C_)
    p["time_w"] = rng.standard_normal((D, T)) / math.sqrt(D)
    p["time_b"] = np.zeros(T)
    p["p1_w"] = rng.standard_normal((C_, Hp)) / math.sqrt(C_)
    p["p1_b"] = np.zeros(Hp)
    p["p2_w"] = rng.standard_normal((Hp, 2)) / math.sqrt(Hp)
    p["p2_b"] = np.zeros(2)
    return {k: v.astype(np.float32) for k, v in p.items()}


class FNO:
    """The network on one GPU: FP32 master weights, BF16 GEMM copies,
    activations for a batch of B shots, forward / backward / Adam through
    the sfg_fno_* kernels."""

    GEMM_WEIGHTS = ("lift_w", "time_w", "p1_w", "p2_w")

    def __init__(self, params: dict, B: int, D: int, W: int, T: int, device, stream=None, layers: int = 4,
                 kernels=None):
        import torch
        self.torch = torch
        self.dev = torch.device(device)
        self.B, self.D, self.W, self.T, self.Lyr = B, D, W, T, layers
        self.C = params["lift_w"].shape[0]
        self.Hp = params["p1_w"].shape[1]
        self.cin = params["lift_w"].shape[1]
        self.K = kernels if kernels is not None else Kernels(stream)
        f32 = dict(dtype=torch.float32, device=self.dev)
        bf = dict(dtype=torch.bfloat16, device=self.dev)
        self.p = {k: torch.tensor(np.ascontiguousarray(v), **f32) for k, v in params.items()}
        # all gradients in one flat buffer: one all-reduce per step for data parallelism
        self.gflat = torch.zeros(sum(v.numel() for v in self.p.values()), **f32)
        self.g, off = {}, 0
        for k, v in self.p.items():
            self.g[k] = self.gflat[off:off + v.numel()].view(v.shape)
            off += v.numel()
        self.m = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.step_count = 0
        Fw, Gd, Gi2, Gw = dft_mats(D, W)
        self.Fw, self.Gd, self.Gi2, self.Gw = (torch.tensor(a, **f32).to(torch.bfloat16) for a in (Fw, Gd, Gi2, Gw))
        Cc, P, modes = self.C, D * W, KD * KC
        self.bf = {k: torch.empty(self.p[k].shape, **bf) for k in self.GEMM_WEIGHTS}
        for l in range(layers):
            self.bf[f"cw{l}"] = torch.empty((Cc, Cc), **bf)
            self.bf[f"wblk{l}"] = torch.empty((modes, 2 * Cc, 2 * Cc), **bf)
        self.refresh_weights()
        BC = B * Cc
        e = torch.empty
        self.v_act = [e((B, Cc, P), **bf) for _ in range(layers + 1)]
        self.pre = [e((B, Cc, P), **bf) for _ in range(layers)]
        self.Zmix = [e((modes, B, 2 * Cc), **bf) for _ in range(layers)]
        self.s = e((B, Cc, P), **f32)
        self.Y1 = e((BC * D, 32), **bf)
        self.Pm = e((BC, 64, 32), **f32)
        self.O = e((BC, 2 * modes), **bf)
        self.Yo = e((BC * D, 32), **bf)
        self.u = e((BC, W, T), **bf)
        self.h1 = e((B, W * T, self.Hp), **bf)
        self.hpre = e((B, W * T, self.Hp), **bf)
        self.y = e((B, 2, W * T), **f32)
        # backward buffers
        self.dy = e((B, 2, W * T), **bf)
        self.dh = e((B, W * T, self.Hp), **f32)
        self.dhpre = e((B, W * T, self.Hp), **bf)
        self.du = e((BC, W, T), **bf)
        self.v4t = e((D, BC, W), **bf)
        self.gact = e((B, Cc, P), **bf)
        self.gf = e((B, Cc, P), **f32)
        self.dpre = e((B, Cc, P), **bf)
        self.dYo = e((BC * D, 32), **bf)
        self.dOf = e((BC, 2 * modes), **f32)
        self.dO = e((BC, 2 * modes), **bf)
        self.dZf = e((modes, B, 2 * Cc), **f32)
        self.dZ = e((modes, B, 2 * Cc), **bf)
        self.dWblk = e((modes, 2 * Cc, 2 * Cc), **f32)
        self.dP = e((BC, 64, 32), **bf)
        self.dY1 = e((BC * D, 32), **bf)
        self.loss = e((B,), **f32)
        self.scratch = e((2 * B,), **f32)

    # ------------------------------------------------------------ weights
    def refresh_weights(self):
        K = self.K
        for k in self.GEMM_WEIGHTS:
            K.call("sfg_fno_cast_bf16", self.p[k], self.bf[k], self.p[k].numel())
        for l in range(self.Lyr):
            K.call("sfg_fno_cast_bf16", self.p[f"cw{l}"], self.bf[f"cw{l}"], self.C * self.C)
            K.call("sfg_fno_expand_weights", self.p[f"wr{l}"], self.p[f"wi{l}"],
                   self.bf[f"wblk{l}"], KD * KC, self.C)

    def params_numpy(self):
        return {k: v.float().cpu().numpy() for k, v in self.p.items()}

    # ------------------------------------------------------------ spectral
    def _spectral(self, l, vin, s):
        K, B, Cc, D, W = self.K, self.B, self.C, self.D, self.W
        BC = B * Cc
        BCD, M5 = BC * D, KD * KC
        K.gemm(vin, self.Fw, self.Y1, BCD, 32, W, a=(0, 0, W, 1), b=(0, 0, 32, 1), c=(0, 0, 32, 1))
        K.gemm(self.Gd, self.Y1, self.Pm, 64, 32, D, a=(0, 0, D, 1), b=(D * 32, 0, 32, 1), c=(2048, 0, 32, 1),
               batch=(BC, 1))
        K.call("sfg_fno_dft_combine", self.Pm, self.Zmix[l], B, Cc)
        wb = self.bf[f"wblk{l}"]
        for ri in (0, 1):
            K.gemm(self.Zmix[l], wb, self.O, B, Cc, 2 * Cc, a=(B * 2 * Cc, 0, 2 * Cc, 1),
                   b=(4 * Cc * Cc, 0, 2 * Cc, 1), boff=ri * Cc, c=(1, 0, Cc * 2 * M5, 2 * M5), coff=ri * M5,
                   batch=(M5, 1))
        for h in (0, 1):
            K.gemm(self.Gi2, self.O, self.Yo, D, 16, 2 * KD, aoff=h * D * 64, a=(0, 0, 64, 1),
                   b=(2 * M5, 0, 16, 1), c=(D * 32, 0, 32, 1), coff=h * 16, batch=(BC, 1))
        K.gemm(self.Yo, self.Gw, s, BCD, W, 32, a=(0, 0, 32, 1), b=(0, 0, W, 1), c=(0, 0, W, 1))

    def _spectral_bwd(self, l, dpre, ds):
        K, B, Cc, D, W = self.K, self.B, self.C, self.D, self.W
        BC = B * Cc
        BCD, M5 = BC * D, KD * KC
        K.gemm(dpre, self.Gw, self.dYo, BCD, 32, W, a=(0, 0, W, 1), b=(0, 0, 1, W), c=(0, 0, 32, 1))
        K.gemm(self.Gi2, self.dYo, self.dOf, 2 * KD, 16, D, a=(0, 0, 1, 64), b=(D * 32, 0, 32, 1),
               c=(2 * M5, 0, 16, 1), batch=(BC, 1))
        K.gemm(self.Gi2, self.dYo, self.dO, 2 * KD, 16, D, aoff=D * 64, boff=16, a=(0, 0, 1, 64),
               b=(D * 32, 0, 32, 1), c=(2 * M5, 0, 16, 1), batch=(BC, 1), Cin=self.dOf)
        wb = self.bf[f"wblk{l}"]
        K.gemm(self.dO, wb, self.dZf, B, 2 * Cc, Cc, a=(1, 0, Cc * 2 * M5, 2 * M5), b=(4 * Cc * Cc, 0, 1, 2 * Cc),
               c=(B * 2 * Cc, 0, 2 * Cc, 1), batch=(M5, 1))
        K.gemm(self.dO, wb, self.dZ, B, 2 * Cc, Cc, aoff=M5, boff=Cc, a=(1, 0, Cc * 2 * M5, 2 * M5),
               b=(4 * Cc * Cc, 0, 1, 2 * Cc), c=(B * 2 * Cc, 0, 2 * Cc, 1), batch=(M5, 1), Cin=self.dZf)
        for ri in (0, 1):
            K.gemm(self.Zmix[l], self.dO, self.dWblk, 2 * Cc, Cc, B, boff=ri * M5, coff=ri * Cc,
                   a=(B * 2 * Cc, 0, 1, 2 * Cc), b=(1, 0, Cc * 2 * M5, 2 * M5), c=(4 * Cc * Cc, 0, 2 * Cc, 1),
                   batch=(M5, 1))
        K.call("sfg_fno_fold_weights", self.dWblk, self.g[f"wr{l}"], self.g[f"wi{l}"], M5, Cc)
        K.call("sfg_fno_dft_combine_bwd", self.dZ, self.dP, B, Cc)
        K.gemm(self.Gd, self.dP, self.dY1, D, 32, 64, a=(0, 0, 1, D), b=(2048, 0, 32, 1), c=(D * 32, 0, 32, 1),
               batch=(BC, 1))
        K.gemm(self.dY1, self.Fw, ds, BCD, W, 32, a=(0, 0, 32, 1), b=(0, 0, 1, 32), c=(0, 0, W, 1))

    # ------------------------------------------------------------ network
    def forward(self, x, keep_pre: bool = True):
        """x: BF16 [B][cin][D][W] on the device -> self.y (FP32 [B][2][W][T]).
        keep_pre=False (inference) skips storing the pre-activations that
        only backward() reads and fuses the two head projections."""
        K, B, Cc, D, W, T, Hp = self.K, self.B, self.C, self.D, self.W, self.T, self.Hp
        P = D * W
        K.gemm(self.bf["lift_w"], x, self.v_act[0], Cc, P, self.cin, a=(0, 0, self.cin, 1),
               b=(self.cin * P, 0, P, 1), c=(Cc * P, 0, P, 1), batch=(B, 1), bias=self.p["lift_b"], bias_on_m=True)
        for l in range(self.Lyr):
            self._spectral(l, self.v_act[l], self.s)
            last = l == self.Lyr - 1
            K.gemm(self.bf[f"cw{l}"], self.v_act[l], self.v_act[l + 1], Cc, P, Cc, a=(0, 0, Cc, 1),
                   b=(Cc * P, 0, P, 1), c=(Cc * P, 0, P, 1), batch=(B, 1), Cin=self.s,
                   bias=self.p[f"cb{l}"], bias_on_m=True, pre=None if (last or not keep_pre) else self.pre[l],
                   gelu=not last)
        # depth -> time: u[z][w][t] = sum_d v4[z][d][w] Wt[d][t] + bt[t]
        K.gemm(self.v_act[self.Lyr], self.bf["time_w"], self.u, W, T, D, a=(D * W, 0, 1, W), b=(0, 0, T, 1),
               c=(W * T, 0, T, 1), batch=(B * Cc, 1), bias=self.p["time_b"])
        # head: inference runs both projections in one kernel (the hidden layer
        # stays on chip, FP32 second projection); training stores h1, hpre
        fused = (not keep_pre and hasattr(K, "head_infer") and
                 K.head_infer(self.u, self.bf["p1_w"], self.y, W * T, Hp, Cc, a=(Cc * W * T, 0, 1, W * T),
                              b=(0, 0, Hp, 1), batch=B, bias=self.p["p1_b"], w2=self.p["p2_w"], b2=self.p["p2_b"],
                              y_batch=2 * W * T, y_ch=W * T))
        if not fused:
            K.gemm(self.u, self.bf["p1_w"], self.h1, W * T, Hp, Cc, a=(Cc * W * T, 0, 1, W * T), b=(0, 0, Hp, 1),
                   c=(W * T * Hp, 0, Hp, 1), batch=(B, 1), bias=self.p["p1_b"], pre=self.hpre if keep_pre else None,
                   gelu=True)
            K.gemm(self.h1, self.bf["p2_w"], self.y, W * T, 2, Hp, a=(W * T * Hp, 0, Hp, 1), b=(0, 0, 2, 1),
                   c=(2 * W * T, 0, 1, W * T), batch=(B, 1), bias=self.p["p2_b"])
        return self.y

    def loss_and_grad(self, target, want_grad=True):
        """Relative-L2 loss per shot against target (BF16 [B][2][W][T]);
        fills self.dy with its gradient."""
        n = 2 * self.W * self.T
        self.K.call("sfg_fno_rel_loss", self.y, target, self.loss,
                    self.dy if want_grad else None, self.scratch, self.B, n)
        return self.loss

    def zero_grad(self):
        self.K.call("sfg_fno_zero", self.gflat, self.gflat.numel())

    def backward(self, x):
        """Gradients of all parameters (into self.g, accumulated) from self.dy."""
        K, B, Cc, D, W, T, Hp = self.K, self.B, self.C, self.D, self.W, self.T, self.Hp
        P, WT, BC = D * W, W * T, B * Cc
        g = self.g
        # head
        K.gemm(self.h1, self.dy, g["p2_w"], Hp, 2, WT, a=(WT * Hp, 0, 1, Hp), b=(2 * WT, 0, 1, WT),
               c=(0, 0, 2, 1), batch=(B, 1), atomic=True, splits=16)
        K.call("sfg_fno_bias_grad", self.dy, g["p2_b"], B, 2, WT)
        K.gemm(self.dy, self.bf["p2_w"], self.dh, WT, Hp, 2, a=(2 * WT, 0, 1, WT), b=(0, 0, 1, 2),
               c=(WT * Hp, 0, Hp, 1), batch=(B, 1))
        K.call("sfg_fno_gelu_bwd", self.dh, 0, self.hpre, self.dhpre, B * WT * Hp)
        K.gemm(self.u, self.dhpre, g["p1_w"], Cc, Hp, WT, a=(Cc * WT, 0, WT, 1), b=(WT * Hp, 0, Hp, 1),
               c=(0, 0, Hp, 1), batch=(B, 1), atomic=True, splits=16)
        K.call("sfg_fno_bias_grad", self.dhpre, g["p1_b"], B * WT, Hp, 1)
        K.gemm(self.dhpre, self.bf["p1_w"], self.du, WT, Cc, Hp, a=(WT * Hp, 0, Hp, 1), b=(0, 0, 1, Hp),
               c=(Cc * WT, 0, 1, WT), batch=(B, 1))
        # time map
        K.call("sfg_fno_swap01", self.v_act[self.Lyr], self.v4t, BC, D, W)
        K.gemm(self.v4t, self.du, g["time_w"], D, T, BC * W, a=(0, 0, BC * W, 1), b=(0, 0, T, 1), c=(0, 0, T, 1),
               atomic=True, splits=32)
        K.call("sfg_fno_bias_grad", self.du, g["time_b"], BC * W, T, 1)
        K.gemm(self.bf["time_w"], self.du, self.gact, D, W, T, a=(0, 0, T, 1), b=(W * T, 0, 1, T),
               c=(D * W, 0, W, 1), batch=(BC, 1))
        # Fourier layers, last to first; self.gact holds dL/dv_{l+1} (BF16)
        for l in reversed(range(self.Lyr)):
            last = l == self.Lyr - 1
            if last:
                dpre = self.gact
            else:
                K.call("sfg_fno_gelu_bwd", self.gact, 1, self.pre[l], self.dpre, B * Cc * P)
                dpre = self.dpre
            vin = self.v_act[l]
            K.gemm(dpre, vin, g[f"cw{l}"], Cc, Cc, P, a=(Cc * P, 0, P, 1), b=(Cc * P, 0, 1, P), c=(0, 0, Cc, 1),
                   batch=(B, 1), atomic=True, splits=8)
            K.call("sfg_fno_bias_grad", dpre, g[f"cb{l}"], B, Cc, P)
            self._spectral_bwd(l, dpre, self.gf)
            K.gemm(self.bf[f"cw{l}"], dpre, self.gact if not last else self.dpre, Cc, P, Cc, a=(0, 0, 1, Cc),
                   b=(Cc * P, 0, P, 1), c=(Cc * P, 0, P, 1), batch=(B, 1), Cin=self.gf)
            if last:   # dpre aliased gact: the new gradient went to dpre
                self.gact, self.dpre = self.dpre, self.gact
        # lift
        K.gemm(self.gact, x, g["lift_w"], Cc, self.cin, P, a=(Cc * P, 0, P, 1), b=(self.cin * P, 0, 1, P),
               c=(0, 0, self.cin, 1), batch=(B, 1), atomic=True, splits=8)
        K.call("sfg_fno_bias_grad", self.gact, g["lift_b"], B, Cc, P)

    def allreduce_grads(self, group=None):
        """Data parallelism: average the gradients over the ranks of `group`
        (torch.distributed: NCCL between GPUs, gloo on CPUs), one all-reduce
        of the flat gradient buffer.  Every rank's loss is the mean over its
        own shots, so the average is the gradient of the mean over all."""
        import torch.distributed as dist
        world = dist.get_world_size(group)
        if world > 1:
            dist.all_reduce(self.gflat, op=dist.ReduceOp.SUM, group=group)
            self.K.call("sfg_fno_scale", self.gflat, self.gflat.numel(), 1.0 / world)

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        for k, p in self.p.items():
            self.K.call("sfg_fno_adam", p, self.g[k], self.m[k], self.v[k], p.numel(),
                        lr, beta1, beta2, eps, self.step_count)
        self.refresh_weights()

    def train_step(self, x, target, lr=1e-3, group=None):
        """One Adam step on this batch; with `group` (data parallelism) the
        gradients are averaged over its ranks first."""
        self.zero_grad()
        self.forward(x)
        self.loss_and_grad(target)
        self.backward(x)
        if group is not None:
            self.allreduce_grads(group)
        self.adam(lr)
        return self.loss


# ------------------------------------------------------------------ data

def features(prob, D: int = 128) -> np.ndarray:
    """Network input [4][D][W] of a config-5 shot: the model on the depth x
    receiver-column grid (depth 0 = the surface row), a Gaussian of the
    source's horizontal position, and the two coordinates."""
    m = prob.mesh
    n = int(round(math.sqrt(m.node_num))) - 1
    h = prob.edge_size
    vp = prob.model.vp.reshape(n + 1, n + 1)                  # [y index][x index]: node = ix + iy (n + 1)
    cols = np.rint(m.y[prob.rec_node] / h).astype(int)        # receiver columns (y)
    rows = n - np.arange(D)                                    # depth d: x = (n - d) h
    W = len(cols)
    x = np.empty((4, D, W), np.float32)
    x[0] = (vp[np.ix_(cols, rows)].T - 3000.0) / 400.0
    ys = m.y[prob.src_node[0]]
    x[1] = np.exp(-(((m.y[prob.rec_node] - ys) / (3 * h)) ** 2))[None, :]
    x[2] = (np.arange(D) / D)[:, None]
    x[3] = (np.arange(W) / W)[None, :]
    return x


def target(seis_u: np.ndarray, seis_w: np.ndarray) -> np.ndarray:
    """The receiver gather [2][W][T] (u, w displacement; receiver-major) from
    the FEM's [T][W] seismograms."""
    return np.stack([seis_u.T, seis_w.T]).astype(np.float32)


def moveout_samples(seeds, speed: float = 3000.0, **cfg) -> np.ndarray:
    """Per shot and receiver [n][W]: the whole samples |y_rec - y_src| / speed
    / dt of a wave at `speed` from the source to each receiver (config-5
    geometry; no FEM run)."""
    from .problem import config_5
    out = []
    for s in seeds:
        p = config_5(int(s), **cfg)
        m = p.mesh
        off = np.abs(m.y[p.rec_node] - m.y[p.src_node[0]])
        out.append(np.floor(off / speed / p.dt).astype(np.int32))
    return np.stack(out)


def to_reduced_time(y: np.ndarray, shift: np.ndarray) -> np.ndarray:
    """y[n][c][W][T] -> the traces advanced by their moveout: r[..., w, tau] =
    y[..., w, tau + shift[n, w]] (zeros past the end).  Exact inverse
    from_reduced_time for every sample at or after the shift; the samples
    before it (ahead of the first arrival at that speed) are dropped."""
    out = np.zeros_like(y)
    T = y.shape[-1]
    for n in range(y.shape[0]):
        for w in range(y.shape[2]):
            s = int(shift[n, w])
            if s < T:
                out[n, :, w, :T - s] = y[n, :, w, s:]
    return out


def from_reduced_time(r: np.ndarray, shift: np.ndarray) -> np.ndarray:
    """Inverse of to_reduced_time: y[..., w, t] = r[..., w, t - shift[n, w]]
    for t >= shift, zero before."""
    out = np.zeros_like(r)
    T = r.shape[-1]
    for n in range(r.shape[0]):
        for w in range(r.shape[2]):
            s = int(shift[n, w])
            if s < T:
                out[n, :, w, s:] = r[n, :, w, :T - s]
    return out


def generate(seeds, device: int = 0, D: int = 128, batch: int = 64, **cfg):
    """FEM shots for `seeds` (config_5; one mesh, each shot its own model and
    source): inputs [n][4][D][W], gathers [n][2][W][T] and the FEM's wall
    time per shot.  Shots advance `batch` at a time through sfg_run_models
    (compensated FP32) in one context set up once on the mesh."""
    import copy
    import time
    from .problem import config_5
    seeds = [int(s) for s in seeds]
    probs = [config_5(s, **cfg) for s in seeds]
    xs = np.stack([features(p, D) for p in probs])
    ys = []
    ctx = api.Context(device)
    t0 = time.perf_counter()        # after the process's CUDA start-up
    ctx.setup(probs[0])
    for k in range(0, len(probs), batch):
        chunk = probs[k:k + batch]
        p = copy.copy(chunk[0])
        p.src_node = np.concatenate([q.src_node for q in chunk]).astype(np.int32)
        r = ctx.run_models(p, [q.model for q in chunk], shots_per_batch=32 if len(chunk) <= 32 else 64)
        ys += [target(r["seis_u"][j], r["seis_w"][j]) for j in range(len(chunk))]
    ctx.close()
    secs = np.full(len(probs), (time.perf_counter() - t0) / max(len(probs), 1))
    return xs, np.stack(ys), secs


def hybrid(err: np.ndarray, bound: float, sur_seconds_per_shot: float, fem_seconds_per_shot: float) -> dict:
    """The surrogate with the FEM as its fallback: every shot runs the
    surrogate, and the shots whose error passes `bound` run the FEM too (an
    exact error judge: the fraction is the best case of any estimate of the
    error).  Returns the fallback fraction and shots per second."""
    fb = np.asarray(err) > bound
    n = len(fb)
    t = n * sur_seconds_per_shot + int(fb.sum()) * fem_seconds_per_shot
    return {"bound": float(bound), "fallback_fraction": float(fb.mean()), "shots_per_s": n / t if t > 0 else 0.0}


def rel_l2(pred: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Per-shot relative L2 error over the whole gather."""
    B = ref.shape[0]
    d = (pred - ref).reshape(B, -1)
    return np.linalg.norm(d, axis=1) / np.maximum(np.linalg.norm(ref.reshape(B, -1), axis=1), 1e-30)


class Surrogate:
    """Training and inference around FNO on one GPU (`device`: a CUDA index,
    or a torch device with `kernels` standing in for the CUDA library).
    Targets are scaled by one global factor (their RMS over the training
    set).  With a torch.distributed `group`, fit() trains data-parallel:
    every rank takes B shots of each global batch of B * ranks and the
    gradients are averaged before each Adam step."""

    def __init__(self, B: int = 16, C_: int = 64, Hp: int = 128, D: int = 128, W: int = 64, T: int = 1000,
                 device=0, seed: int = 0, stream=None, kernels=None):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        self.B, self.D, self.W, self.T = B, D, W, T
        self.net = FNO(init_params(C_, D, T, Hp, seed=seed), B, D, W, T, self.dev, stream=stream, kernels=kernels)
        self.scale = 1.0

    def _batch(self, arr, idx, dtype):
        t = self.torch.tensor(arr[idx], dtype=self.torch.float32)
        return t.to(self.dev).to(dtype).contiguous()

    def fit(self, x: np.ndarray, y: np.ndarray, epochs: int, lr: float = 2e-3, seed: int = 0, log=None,
            group=None):
        """Adam on the relative-L2 loss; returns the mean loss per epoch (over
        all ranks' shots).  Every rank passes the same x, y and seed; with
        `group`, rank r trains on shots [r B, (r + 1) B) of each global batch
        of the epoch's permutation."""
        torch = self.torch
        rank, world = 0, 1
        if group is not None:
            import torch.distributed as dist
            rank, world = dist.get_rank(group), dist.get_world_size(group)
        self.scale = float(np.sqrt(np.mean(y.astype(np.float64) ** 2))) or 1.0
        G = self.B * world
        n = (len(x) // G) * G
        xd = torch.tensor(x[:n]).to(self.dev).to(torch.bfloat16)
        yd = (torch.tensor(y[:n]) / self.scale).to(self.dev).to(torch.bfloat16)
        rng = np.random.default_rng(seed)
        hist = []
        steps = epochs * (n // G)
        it = 0
        for ep in range(epochs):
            perm = rng.permutation(n)
            tot = torch.zeros(1, dtype=torch.float64)
            for k in range(0, n, G):
                idx = torch.tensor(perm[k + rank * self.B:k + (rank + 1) * self.B], device=self.dev)
                xb = xd.index_select(0, idx).contiguous()
                yb = yd.index_select(0, idx).contiguous()
                # cosine learning-rate decay
                lr_t = lr * 0.5 * (1 + math.cos(math.pi * it / max(steps, 1)))
                loss = self.net.train_step(xb, yb, lr_t, group=group if world > 1 else None)
                tot += float(loss.sum().item())
                it += 1
            if world > 1:
                import torch.distributed as dist
                tot = tot.to(self.dev) if dist.get_backend(group) == "nccl" else tot
                dist.all_reduce(tot, group=group)
            hist.append(float(tot.item()) / n)
            if log:
                log(f"epoch {ep}: loss {hist[-1]:.4f}")
        return hist

    def inference_net(self, batch: int):
        """The network with the current weights for `batch` shots per pass
        (larger batches make larger GEMMs; the training batch is self.B)."""
        if batch == self.B:
            return self.net
        key = (batch, self.net.step_count)
        if getattr(self, "_infer", (None, None))[0] != key:
            self._infer = (key, FNO(self.net.params_numpy(), batch, self.D, self.W, self.T, self.dev,
                                    stream=self.net.K.stream, kernels=None if isinstance(self.net.K, Kernels)
                                    else self.net.K))
        return self._infer[1]

    def predict(self, x: np.ndarray, batch: int | None = None) -> np.ndarray:
        """Gathers [n][2][W][T] (physical units) for inputs [n][4][D][W],
        `batch` shots per forward pass (default: the training batch)."""
        torch = self.torch
        net = self.inference_net(batch or self.B)
        Bp = net.B
        out = np.empty((len(x), 2, self.W, self.T), np.float32)
        for k in range(0, len(x), Bp):
            xb = np.zeros((Bp, 4, self.D, self.W), np.float32)
            m = min(Bp, len(x) - k)
            xb[:m] = x[k:k + m]
            y = net.forward(torch.tensor(xb).to(self.dev).to(torch.bfloat16).contiguous(), keep_pre=False)
            out[k:k + m] = y[:m].float().cpu().numpy().reshape(m, 2, self.W, self.T) * self.scale
        return out
