"""The learned surrogate: its kernels against FP32 references, its gradients
against the CPU oracle (oracle/fno_oracle.py, torch autograd with torch.fft
spectral convolutions), and a trained network against the untrained one and
the zero predictor on held-out FEM shots."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from seisfem_b200.surrogate import FNO, dft_mats, init_params  # noqa: E402

SMALL = dict(B=2, D=32, W=32, T=48, C=8, Hp=16)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _case(seed=0):
    import torch
    s = SMALL
    prm = init_params(s["C"], s["D"], s["T"], s["Hp"], seed=seed + 1)
    rng = np.random.default_rng(seed)
    x = torch.tensor(rng.standard_normal((s["B"], 4, s["D"], s["W"])).astype(np.float32)).to(torch.bfloat16)
    t = torch.tensor(rng.standard_normal((s["B"], 2, s["W"], s["T"])).astype(np.float32)).to(torch.bfloat16)
    return prm, x, t


def _run(net, x, t):
    net.zero_grad()
    y = net.forward(x).float().cpu().numpy().copy()
    loss = net.loss_and_grad(t).float().cpu().numpy().copy()
    net.backward(x)
    return y, loss, {k: v.float().cpu().numpy() for k, v in net.g.items()}


def test_dft_matrices_invert_kept_modes():
    # forward then inverse of a signal made of kept modes only is the identity
    D, W = 32, 32
    Fw, Gd, Gi2, Gw = dft_mats(D, W)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((D, W))
    X = np.fft.rfft2(x)
    keep = np.zeros_like(X)
    keep[:16, :16] = X[:16, :16]
    keep[D - 16:, :16] = X[D - 16:, :16]
    xk = np.fft.irfft2(keep, s=(D, W))
    Y1 = xk @ Fw                                   # [D][32]
    P = Gd @ Y1                                    # [64][32]
    Zre = P[:32, :16] + P[32:, 16:]
    Zim = P[:32, 16:] - P[32:, :16]
    assert np.allclose(Zre + 1j * Zim, np.concatenate([keep[:16, :16], keep[D - 16:, :16]]), atol=1e-9)
    O = np.concatenate([Zre, Zim])                 # [64][16]
    Yo = np.concatenate([Gi2[:D] @ O, Gi2[D:] @ O], axis=1)
    assert np.allclose(Yo @ Gw, xk, atol=1e-9)


def test_host_sequencing_matches_oracle_on_cpu():
    """Every stride and layout of the surrogate's GEMM sequence, run through
    a CPU emulation of the kernels, against the FP32 oracle."""
    import fno_oracle
    from fno_emulator import EmuKernels
    s = SMALL
    prm, x, t = _case()
    y_ref, l_ref, g_ref = fno_oracle.loss_and_grads(prm, x.float().numpy(), t.float().numpy())
    net = FNO(prm, s["B"], s["D"], s["W"], s["T"], "cpu", kernels=EmuKernels())
    y, loss, g = _run(net, x, t)
    assert _rel(y.reshape(y_ref.shape), y_ref) < 2e-2
    assert np.allclose(loss, l_ref, rtol=1e-2)
    for k in prm:
        assert _rel(g[k], g_ref[k]) < 3e-2, k


# ------------------------------------------------------------------ GPU

@pytest.mark.gpu
@pytest.mark.parametrize("engine", [1, 2, 3, 4])
@pytest.mark.parametrize("layout", ["nn", "tn", "nt", "strided"])
def test_gemm_matches_fp32(layout, engine):
    """Every epilogue term (alpha, beta Cin, bias, stored pre-activation,
    GELU) on both engines; odd strides take the mma.sync engine."""
    import torch
    from seisfem_b200.surrogate import Kernels
    K = Kernels()
    K.engine = engine
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(3)
    b1, b2, M, N, Kd = 3, 2, 150, 70, 90
    A = torch.tensor(rng.standard_normal((b1, b2, M, Kd)).astype(np.float32)).to(torch.bfloat16)
    B = torch.tensor(rng.standard_normal((b1, b2, Kd, N)).astype(np.float32)).to(torch.bfloat16)
    bias = torch.tensor(rng.standard_normal(N).astype(np.float32))
    Cin = torch.tensor(rng.standard_normal((b1, b2, M, N)).astype(np.float32))
    ref = torch.nn.functional.gelu(A.float() @ B.float() * 0.5 + 2.0 * Cin + bias)
    if layout in ("tn", "strided"):
        Ad = A.transpose(2, 3).contiguous().to(dev)          # stored [b1][b2][K][M]
        sa = (b2 * Kd * M, Kd * M, 1, M)
    else:
        Ad = A.contiguous().to(dev)
        sa = (b2 * M * Kd, M * Kd, Kd, 1)
    if layout in ("nt", "strided"):
        Bd = B.transpose(2, 3).contiguous().to(dev)          # stored [b1][b2][N][K]
        sb = (b2 * N * Kd, N * Kd, 1, Kd)
    else:
        Bd = B.contiguous().to(dev)
        sb = (b2 * Kd * N, Kd * N, N, 1)
    if layout == "strided":   # odd strides: the scalar load path
        Ad2 = torch.zeros(b1 * b2 * M * Kd * 3, dtype=torch.bfloat16, device=dev)
        Ad2[::3] = Ad.reshape(-1)
        Ad, sa = Ad2, tuple(3 * v for v in sa)
    C = torch.empty((b1, b2, M, N), dtype=torch.float32, device=dev)
    pre = torch.empty((b1, b2, M, N), dtype=torch.bfloat16, device=dev)
    K.gemm(Ad, Bd, C, M, N, Kd, a=sa, b=sb, c=(b2 * M * N, M * N, N, 1), batch=(b1, b2), Cin=Cin.to(dev),
           beta=2.0, alpha=0.5, bias=bias.to(dev), gelu=True, pre=pre)
    torch.cuda.synchronize()
    assert _rel(C.cpu().numpy(), ref.numpy()) < 2e-3
    pre_ref = A.float() @ B.float() * 0.5 + 2.0 * Cin + bias
    assert _rel(pre.float().cpu().numpy(), pre_ref.numpy()) < 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("N,Kd,layout", [(32, 64, "nn"), (64, 100, "tn"), (128, 300, "nt"), (200, 128, "nn"),
                                         (136, 72, "tt"), (40, 200, "tt"), (96, 64, "strided")])
def test_tcgen05_gemm_matches_mma_sync(N, Kd, layout):
    """The tcgen05/TMEM engines -- persistent with TMA tiles (2), cp.async
    tiles (3), TMA tiles one output tile per CTA (4) -- against the mma.sync
    engine on the same descriptor (all accumulate in FP32), incl. ragged M,
    N, K and every load path; no bounded wait may give up."""
    import ctypes
    import torch
    from seisfem_b200.surrogate import Kernels
    K = Kernels()
    dev = torch.device("cuda:0")
    cnt = ctypes.c_int()
    assert K.L.sfg_fno_tc_timeouts(ctypes.byref(cnt), 1) == 0
    rng = np.random.default_rng(N + Kd)
    b1, M = 2, 300
    A = torch.tensor(rng.standard_normal((b1, M, Kd)).astype(np.float32)).to(torch.bfloat16)
    B = torch.tensor(rng.standard_normal((b1, Kd, N)).astype(np.float32)).to(torch.bfloat16)
    bias = torch.tensor(rng.standard_normal(N).astype(np.float32), device=dev)
    if layout in ("tn", "tt", "strided"):       # A m-contiguous: the MN-major tile layout
        Ad, sa = A.transpose(1, 2).contiguous().to(dev), (Kd * M, 0, 1, M)
    else:
        Ad, sa = A.contiguous().to(dev), (M * Kd, 0, Kd, 1)
    if layout in ("nt", "tt"):                  # B k-contiguous: the K-major tile layout
        Bd, sb = B.transpose(1, 2).contiguous().to(dev), (N * Kd, 0, 1, Kd)
    else:
        Bd, sb = B.contiguous().to(dev), (Kd * N, 0, N, 1)
    if layout == "strided":
        Ad2 = torch.zeros(Ad.numel() * 3, dtype=torch.bfloat16, device=dev)
        Ad2[::3] = Ad.reshape(-1)
        Ad, sa = Ad2, tuple(3 * v for v in sa)
    outs = []
    for eng in (1, 2, 3, 4):
        C = torch.empty((b1, M, N), dtype=torch.float32, device=dev)
        K.gemm(Ad, Bd, C, M, N, Kd, a=sa, b=sb, c=(M * N, 0, N, 1), batch=(b1, 1), bias=bias, gelu=True,
               engine=eng)
        outs.append(C.cpu().numpy())
    torch.cuda.synchronize()
    assert K.L.sfg_fno_tc_timeouts(ctypes.byref(cnt), 1) == 0 and cnt.value == 0
    ref = torch.nn.functional.gelu(A.float() @ B.float() + bias.cpu()).numpy()
    for o in outs[1:]:
        assert _rel(o, outs[0]) < 1e-5
        assert _rel(o, ref) < 2e-3


@pytest.mark.gpu
@pytest.mark.parametrize("engine", [1, 2, 3, 4])
def test_gemm_split_k_and_batch_sum(engine):
    import torch
    from seisfem_b200.surrogate import Kernels
    K = Kernels()
    K.engine = engine
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(4)
    b, M, N, Kd = 4, 64, 48, 5000
    A = torch.tensor(rng.standard_normal((b, M, Kd)).astype(np.float32)).to(torch.bfloat16)
    B = torch.tensor(rng.standard_normal((b, Kd, N)).astype(np.float32)).to(torch.bfloat16)
    ref = (A.float() @ B.float()).sum(0)
    C = torch.zeros((M, N), dtype=torch.float32, device=dev)
    K.gemm(A.to(dev), B.to(dev), C, M, N, Kd, a=(M * Kd, 0, Kd, 1), b=(Kd * N, 0, N, 1), c=(0, 0, N, 1),
           batch=(b, 1), atomic=True, splits=7)
    torch.cuda.synchronize()
    assert _rel(C.cpu().numpy(), ref.numpy()) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("engine", [0, 1, 2])
def test_gpu_forward_and_gradients_match_oracle(engine):
    """Engine 0 picks per GEMM, 1 is mma.sync throughout, 2 takes tcgen05
    for every GEMM it can."""
    import torch
    import fno_oracle
    from fno_emulator import EmuKernels
    s = SMALL
    prm, x, t = _case(seed=2)
    y_ref, l_ref, g_ref = fno_oracle.loss_and_grads(prm, x.float().numpy(), t.float().numpy())
    dev = torch.device("cuda:0")
    net = FNO(prm, s["B"], s["D"], s["W"], s["T"], dev)
    net.K.engine = engine
    y, loss, g = _run(net, x.to(dev), t.to(dev))
    torch.cuda.synchronize()
    emu = FNO(prm, s["B"], s["D"], s["W"], s["T"], "cpu", kernels=EmuKernels())
    ye, le, ge = _run(emu, x, t)
    assert _rel(y.reshape(y_ref.shape), y_ref) < 2e-2
    assert np.allclose(loss, l_ref, rtol=1e-2)
    assert _rel(y, ye) < 1e-2
    for k in prm:
        assert _rel(g[k], g_ref[k]) < 3e-2, k
        assert _rel(g[k], ge[k]) < 2e-2, k


@pytest.mark.gpu
@pytest.mark.parametrize("C", [8, 32, 64])
def test_dft_recombination_kernels(C):
    """Forward and backward recombination of the D-DFT outputs (tiled
    kernels for C a multiple of 16, the element-wise ones otherwise)
    against the CPU emulation."""
    import torch
    from fno_emulator import EmuKernels
    from seisfem_b200.surrogate import Kernels
    K, E = Kernels(), EmuKernels()
    B = 3
    rng = np.random.default_rng(C)
    P = torch.tensor(rng.standard_normal((B * C, 64, 32)).astype(np.float32))
    Zc = torch.zeros(512 * B * 2 * C, dtype=torch.bfloat16)
    E.dft_combine(P, Zc, B, C)
    Zg = torch.zeros_like(Zc, device="cuda:0")
    K.call("sfg_fno_dft_combine", P.to("cuda:0"), Zg, B, C)
    dZ = torch.tensor(rng.standard_normal(512 * B * 2 * C).astype(np.float32)).to(torch.bfloat16)
    dPc = torch.zeros((B * C, 64, 32), dtype=torch.bfloat16)
    E.dft_combine_bwd(dZ, dPc, B, C)
    dPg = torch.zeros_like(dPc, device="cuda:0")
    K.call("sfg_fno_dft_combine_bwd", dZ.to("cuda:0"), dPg, B, C)
    torch.cuda.synchronize()
    assert torch.equal(Zg.cpu(), Zc)
    assert torch.equal(dPg.cpu(), dPc)


@pytest.mark.gpu
@pytest.mark.parametrize("hp", [16, 128])
def test_inference_forward_matches_training_forward(hp):
    """keep_pre=False skips the stores backward() reads and, where the
    layout fits (hidden width <= 128, 128-row head tiles), runs the head as
    one kernel with the hidden layer kept in FP32 instead of BF16: equal up
    to that rounding, and against the FP32 oracle."""
    import torch
    import fno_oracle
    s = SMALL
    prm = init_params(s["C"], s["D"], s["T"], hp, seed=5)
    rng = np.random.default_rng(4)
    x = torch.tensor(rng.standard_normal((s["B"], 4, s["D"], s["W"])).astype(np.float32)).to(torch.bfloat16)
    net = FNO(prm, s["B"], s["D"], s["W"], s["T"], torch.device("cuda:0"))
    xd = x.to("cuda:0")
    a = net.forward(xd).float().cpu().numpy().copy()
    b = net.forward(xd, keep_pre=False).float().cpu().numpy().copy()
    assert _rel(b, a) < 1e-2
    t = torch.zeros((s["B"], 2, s["W"], s["T"]), dtype=torch.bfloat16)
    y_ref, _, _ = fno_oracle.loss_and_grads(prm, x.float().numpy(), t.float().numpy())
    assert _rel(b.reshape(y_ref.shape), y_ref) < 2e-2


@pytest.mark.gpu
def test_adam_step_matches_reference_formula():
    import torch
    from seisfem_b200.surrogate import Kernels
    K = Kernels()
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(5)
    p0, g = rng.standard_normal(1000).astype(np.float32), rng.standard_normal(1000).astype(np.float32)
    p, gd = torch.tensor(p0, device=dev), torch.tensor(g, device=dev)
    m, v = torch.zeros(1000, device=dev), torch.zeros(1000, device=dev)
    for step in (1, 2):
        K.call("sfg_fno_adam", p, gd, m, v, 1000, 1e-2, 0.9, 0.999, 1e-8, step)
    torch.cuda.synchronize()
    mm = (1 - 0.9) * g
    vv = (1 - 0.999) * g * g
    q = p0 - 1e-2 * (mm / 0.1) / (np.sqrt(vv / 0.001) + 1e-8)
    mm = 0.9 * mm + 0.1 * g
    vv = 0.999 * vv + 0.001 * g * g
    q = q - 1e-2 * (mm / (1 - 0.81)) / (np.sqrt(vv / (1 - 0.999 ** 2)) + 1e-8)
    assert np.allclose(p.cpu().numpy(), q, rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_trained_surrogate_beats_untrained_on_held_out_fem_shots():
    """64 FEM training shots, 16 held out (config-5 mesh, 200 samples): the
    trained network's mean relative L2 error is well below the untrained
    network's and below the zero predictor's (1.0).  (Its speed against the
    FEM is measured by bench.py's surrogate workload.)"""
    from seisfem_b200.surrogate import Surrogate, generate, rel_l2
    cfg = dict(samples=200)
    xtr, ytr, _ = generate(range(5000, 5064), **cfg)
    xte, yte, _ = generate(range(9000, 9016), **cfg)
    sg = Surrogate(B=8, T=200, seed=0)
    sg.scale = float(np.sqrt(np.mean(ytr.astype(np.float64) ** 2)))
    e0 = rel_l2(sg.predict(xte), yte).mean()
    hist = sg.fit(xtr, ytr, epochs=40, lr=2e-3)
    assert hist[-1] < hist[0]
    pred = sg.predict(xte)
    e1 = rel_l2(pred, yte).mean()
    assert e1 < 0.8 * e0 and e1 < 1.0, (e0, e1)
    # a larger inference batch: the same per-shot arithmetic
    assert _rel(sg.predict(xte, batch=16), pred) < 1e-5


@pytest.mark.gpu
def test_hybrid_beats_the_fem_at_the_error_it_meets():
    """The surrogate with the FEM as fallback, at a stated error: trained on
    128 FEM shots (config-5 mesh, 200 samples, reduced time), judged on 32
    held out.  At the bound the held-out median meets (half the shots fall
    back) the hybrid's shots/s -- surrogate on every shot, FEM on the
    fallen-back ones, per-shot times measured here -- is above the FEM's
    alone; at 1e-2 every shot falls back and the hybrid is slower."""
    import time
    import torch
    from seisfem_b200.surrogate import (Surrogate, from_reduced_time, generate, hybrid, moveout_samples, rel_l2,
                                        to_reduced_time)
    cfg = dict(samples=200)
    xtr, ytr, fem_tr = generate(range(5000, 5128), **cfg)
    xte, yte, _ = generate(range(9000, 9032), **cfg)
    sh_tr, sh_te = moveout_samples(range(5000, 5128), **cfg), moveout_samples(range(9000, 9032), **cfg)
    sg = Surrogate(B=16, T=200, seed=0)
    sg.fit(xtr, to_reduced_time(ytr, sh_tr), epochs=30, lr=2e-3)
    sg.predict(xte)                              # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pred = from_reduced_time(sg.predict(xte), sh_te)
    torch.cuda.synchronize()
    t_sur = (time.perf_counter() - t0) / len(xte)
    t_fem = float(fem_tr[-1])
    err = rel_l2(pred, yte)
    bound = float(np.median(err))
    h = hybrid(err, bound, t_sur, t_fem)
    assert h["fallback_fraction"] <= 0.5 and h["shots_per_s"] > 1.0 / t_fem, (bound, h, 1.0 / t_fem)
    h1 = hybrid(err, 1e-2, t_sur, t_fem)
    assert h1["fallback_fraction"] == 1.0 and h1["shots_per_s"] < 1.0 / t_fem


def test_reduced_time_round_trip():
    """The surrogate's reduced-time targets: every sample at or after a
    trace's moveout comes back exactly; earlier samples (ahead of the first
    arrival at that speed) are zero."""
    from seisfem_b200.surrogate import from_reduced_time, moveout_samples, to_reduced_time
    rng = np.random.default_rng(3)
    y = rng.standard_normal((4, 2, 6, 50)).astype(np.float32)
    sh = rng.integers(0, 60, (4, 6))          # shifts past the trace's end included
    z = from_reduced_time(to_reduced_time(y, sh), sh)
    for n in range(4):
        for w in range(6):
            s = sh[n, w]
            assert np.array_equal(z[n, :, w, s:], y[n, :, w, s:])
            assert not z[n, :, w, :s].any()
    m = moveout_samples([5000, 5001], samples=100, nrec=16)
    assert m.shape == (2, 16) and (m >= 0).all() and m.max() < 500
