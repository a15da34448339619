"""Benchmark of the mass-lumped explicit time loop (DOF-steps/s).

One bench "step" is one complete simulation of the workload -- every time
step of one shot (or one batch of shots) -- with the mesh, matrices and state
resident in HBM.  Default workload: the Q9 400x400 layered model (641,601
nodes, 1,283,202 DOF, 3000 time steps, M-PML 30), FP32 with compensated
displacement.  With N ranks (torchrun, one GPU each) every rank advances its
own shot (shots are independent; no collective inside the loop) and the
job's value is all ranks' DOF-steps over the slowest rank's time.

Printed JSON line: value (device-resident loop), e2e (the public C-ABI call
with host buffers: GPU assembly + run + copies back), roofline of the fused
step kernel, clocks, the CPU baseline (rank 0, N=1), launch counts.
`--impl reference` times the reference's own CPU code (oracle/_ref, else the
oracle port) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from seisfem_b200 import problem as P  # noqa: E402

METRIC = "DOF-steps/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "step_kernel_traffic.txt")
T6_STABLE_STEPS = 602
DEFAULT_WORKLOAD = "q9_400_layered"


def workload(name: str, shots: int = 1):
    if name == "q9_400_layered":
        p = P.config_2()
    elif name == "q4_200_homog":
        p = P.config_1()
    elif name == "q4_400_grf_64shots":
        p = P.config_3a()
    elif name == "t6_300x150_topo_vti":
        # inside the window before the reference's T6 energy bound trips
        p = P.config_4(step=T6_STABLE_STEPS)
    elif name == "q4_200_grf_64shots":
        # the batched kernels on a smaller mesh (profiling case; state > L2)
        p = P.config_3a(n=200, step=500)
    elif name == "q4_200_consistent":
        # config 1's mesh and model through the consistent-mass branch (solver
        # "mgmres"), at dt = 0.5 ms, inside that scheme's stability limit
        p = P.config_1(step=2002)
        p.dt = 5e-4
        p.name = "config1_q4_200_consistent_mass_dt0.5ms"
    else:
        raise SystemExit(f"unknown workload {name}")
    if shots > 1 and len(p.src_node) == 1:
        # a shot list for several ranks: the source moves one element per shot
        m = p.mesh
        x0, y0 = m.x[p.src_node[0]], m.y[p.src_node[0]]
        p.src_node = P.locate(m, p.edge_size, [(x0, y0 + p.edge_size * k) for k in range(shots)])
    return p


def clocks_start(path):
    try:
        f = open(path, "w")
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                stdout=f, stderr=subprocess.DEVNULL), f
    except Exception:
        return None, None


def clocks_stop(proc, f, path, device):
    if proc is None:
        return None
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except Exception:
        proc.kill()
    f.close()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
        parts = [x.strip() for x in line.split(",")]
        if len(parts) < 9 or parts[0] != str(device):
            continue
        try:
            sm.append(float(parts[1]))
            mx = float(parts[2])
        except ValueError:
            continue
        for n, v in zip(names, parts[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(prob_name: str, seconds_budget: float = 30.0, solver: str = "masslump", nsteps: int = 8) -> dict:
    """The reference's own CPU loop (oracle/_ref) on this host's cores, on a
    bounded sample: the full set-up plus a few time steps of the workload,
    each step timed from the reference's end-of-step output."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    prob = workload(prob_name)
    cores = os.cpu_count() or 1
    prob.step = 2 + nsteps
    if os.path.exists(O.LIBREF):
        ref = O.Reference()
        out = ref.run(prob, nthreads=cores, want_snapshots=False, solver=solver)
        t = out["step_end_times"]
        dts = np.diff(t)
        per_step = float(np.median(dts)) if len(dts) else float("nan")
        kind = "reference"
        sample = (f"{prob.name}: reference elastic_wave() solver {solver} with step={prob.step} ({nsteps} time steps, "
                  f"set-up {t[0] - (t[1] - t[0]) if len(t) > 1 else float('nan'):.1f} s excluded); "
                  f"median of per-step times from its end-of-step seismogram writes")
    else:
        orc = O.Oracle()
        out = orc.run(prob, nthreads=cores, solver=solver)
        per_step = out["loop_seconds"] / nsteps
        kind = "port"
        sample = f"{prob.name}: oracle port, {nsteps} time steps, loop time only"
    dof_steps = 2 * prob.mesh.node_num
    return {"value": dof_steps / per_step, "unit": METRIC, "cores": cores, "kind": kind, "sample": sample,
            "seconds_per_step": per_step}


def bench_config(prob, shots_per_rank: int, world: int) -> dict:
    """The workload's description, shared by both arms so that their config
    objects are identical: what is simulated, not how."""
    return {"workload": prob.name, "element": prob.mesh.type_name, "nodes": prob.mesh.node_num,
            "dof": prob.dof, "shots_per_rank": shots_per_rank, "time_steps": prob.step - 2,
            "l2": "per-step working set (matrix + state) > 126 MB L2; no flush needed",
            "parallelism": f"shots over {world} GPU(s)"}


def mapped_repo_libraries() -> list:
    """Shared objects of this repository mapped into this process."""
    out = set()
    try:
        for line in open("/proc/self/maps"):
            f = line.split()
            if len(f) >= 6 and f[-1].endswith(".so") and f[-1].startswith(ROOT):
                out.add(os.path.relpath(f[-1], ROOT))
    except OSError:
        pass
    return sorted(out)


def run_reference_arm(args):
    """The reference's own elastic_wave() (oracle/_ref, compiled from the
    reference sources; else the oracle port) on the host cores.  Its problem
    is built with the numpy node scan, so this process never loads
    libseisfem_b200.so (checked below)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    P.use_scan_locator()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    prob = workload(args.workload)
    cfg = bench_config(prob, len(prob.src_node), args.gpus)
    cores = os.cpu_count() or 1
    n = args.warmup + args.steps
    prob.step = 2 + n
    prob.src_node = prob.src_node[:1]
    if os.path.exists(O.LIBREF):
        solver = "mgmres" if args.workload == "q4_200_consistent" else "masslump"
        out = O.Reference().run(prob, nthreads=cores, want_snapshots=False, solver=solver)
        t = out["step_end_times"]
        dts = np.diff(np.concatenate([[t[0] - (t[1] - t[0])], t])) if len(t) > 1 else np.array([np.nan])
        timed = dts[args.warmup:args.warmup + args.steps]
        kind = "reference"
    else:
        out = O.Oracle().run(prob, nthreads=cores)
        timed = np.full(args.steps, out["loop_seconds"] / n)
        kind = "port"
    ms = float(np.sum(timed)) * 1e3
    # every shot of the workload costs the same per time step; one is timed
    value = 2 * prob.mesh.node_num * args.steps / (ms / 1e3)
    sample = (f"{prob.name}: {n} time steps of one shot of the reference elastic_wave() loop on {cores} host "
              f"threads; bench step = one time step; the first {args.warmup} are warm-up")
    libs = mapped_repo_libraries()
    assert "seisfem_b200.api" not in sys.modules and not any(l.startswith("seisfem_b200") for l in libs), libs
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg,
            "run": {"precision": "fp64 (the reference's own C)", "time_steps_per_bench_step": 1,
                    "repo_libraries_loaded": libs},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


ACOUSTIC_WORKLOADS = {"acoustic_pml_q4_800": dict(n=800, pml=True), "acoustic_q4_800": dict(n=800, pml=False)}


def acoustic_bytes(N: int, union_nnz: int, pml: bool) -> int:
    """Algorithmic bytes of one fused acoustic time step (FP64): per union
    entry its column (4 B) and matrix values (M, K0: 16 B; M, K1, K5, K2, K6:
    40 B); per node its row length (4 B), coefficients ((vp dt)^2 and the
    lumped mass, plus four PML profiles), one read of each gathered state
    vector (u_now, u_old; or u1 now/old, u2 now/old, p1, p2, u) and the
    written vectors (u; or u1, u2, p1, p2, u)."""
    if pml:
        return union_nnz * (4 + 40) + N * (4 + 6 * 8 + 7 * 8 + 5 * 8)
    return union_nnz * (4 + 16) + N * (4 + 2 * 8 + 2 * 8 + 8)


def run_acoustic(args):
    """The scalar acoustic solvers (sfg_acoustic_run): one bench step = one
    complete run (assembly on the GPU, time loop, outputs copied back).
    value: node-steps per second of the time loop (CUDA events around the
    loop's graph launch inside the library); e2e: the same work over the
    wall time of the whole C-ABI call with host arrays in and out."""
    import torch
    from seisfem_b200.api import Context
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    c = P.acoustic_grf(**ACOUSTIC_WORKLOADS[args.workload])
    m, N, steps = c.mesh, c.mesh.node_num, c.step - 2
    n_el = ACOUSTIC_WORKLOADS[args.workload]["n"]
    ctx = Context(0)
    run = lambda: ctx.acoustic_run(m, c.vp, c.step, c.dt, c.f0, 0.0, c.src, c.pml, c.edge_size, c.pml_n, c.pml_n)
    for _ in range(args.warmup):
        r = run()
    assert r["status"] == 0, r["status"]
    cpath = os.path.join(tempfile.gettempdir(), "sfg_clocks_acoustic.csv")
    cproc, cf = clocks_start(cpath)
    loop_ms, wall = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = run()
        wall.append(time.perf_counter() - t0)
        loop_ms.append(r["stats"]["loop_ms"])
    clocks = clocks_stop(cproc, cf, cpath, 0)
    st = r["stats"]
    ms = float(np.sum(loop_ms)) / args.steps
    value = N * steps / (ms * 1e-3)
    b_step = acoustic_bytes(N, st["union_nnz"], c.pml)
    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = b_step * steps / (ms * 1e-3) / 1e9
    rows = r["snap"].shape[0]
    line = {"metric": "node-steps/s", "value": value, "unit": "node-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": c.name, "nodes": N, "elements": f"Q4 {n_el}x{n_el}",
                       "time_steps": steps, "pml": c.pml, "solver": "acoustic_pml.c" if c.pml else "acoustic.c",
                       "l2": "per-step working set > 126 MB L2" if b_step > 126e6 else "per-step working set fits L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "algorithmic_bytes_per_step": b_step},
            "e2e": {"value": N * steps / float(np.mean(wall)), "unit": "node-steps/s",
                    "h2d_bytes_per_step": int(m.element_node.nbytes + 3 * 8 * N),
                    "d2h_bytes_per_step": int(rows * N * 8 + c.step * 8)},
            "setup_ms": st["setup_ms"], "gpu_launches": st["kernel_launches"] * args.steps, "clocks": clocks,
            "cpu_baseline": None}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = acoustic_reference(c, nsteps=24)
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def acoustic_reference(c, nsteps: int) -> dict:
    """The reference's acoustic solver (oracle/_ref, else the oracle port) on
    this host's cores, on a bounded sample of the workload: nsteps time steps
    after its set-up, each timed from its end-of-step energy.dat write."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    m, N = c.mesh, c.mesh.node_num
    if os.path.exists(O.LIBACOUSTIC):
        out = O.ReferenceAcoustic().run(m, c.vp, 2 + nsteps, c.dt, c.f0, 0.0, c.src, c.pml, c.edge_size, c.pml_n,
                                        c.pml_n, nthreads=cores)
        per_step = float(np.median(out["step_seconds"]))
        kind, what = "reference", "reference acoustic_pml()" if c.pml else "reference acoustic()"
    else:
        t0 = time.perf_counter()
        O.Oracle().acoustic_run(m, c.vp, 2 + nsteps, c.dt, c.f0, 0.0, c.src, c.pml, c.edge_size, c.pml_n,
                                c.pml_n, nthreads=cores)
        per_step = (time.perf_counter() - t0) / nsteps
        kind, what = "port", "oracle port (set-up included)"
    return {"value": N / per_step, "unit": "node-steps/s", "cores": cores, "kind": kind,
            "sample": f"{c.name}: {what}, {nsteps} time steps on {cores} host threads; median per-step time",
            "seconds_per_step": per_step}


def consistent_bytes(N: int, union_nnz: int, steps: int, iterations: int) -> int:
    """Algorithmic bytes of a consistent-mass run (FP64): per time step the
    right-hand-side kernel (the union pattern with 7 FP64 values and its
    column, the 20-value state record and 12 coefficients read, 14 values
    written) and the Newmark kernel (14 solved values, 20 + 12 state values
    read and written); per conjugate-gradient iteration q = M p (M's
    column and value, p read and q written, 14 columns), the update (x, p,
    q, r read; x, r, z written; 1/diag) and the new directions (z, p read,
    p written)."""
    per_step = union_nnz * (4 + 7 * 8) + N * 8 * (20 + 12 + 14) + N * 8 * (14 + 2 * (20 + 12))
    per_iter = union_nnz * (4 + 8) + N * 8 * (14 * (2 + 7 + 3) + 1)
    return steps * per_step + iterations * per_iter


def run_consistent(args):
    """The consistent-mass branch (SFG_FP64_CONSISTENT): one bench step = one
    complete simulation of the workload, device-resident (CUDA events around
    the plan's launch); e2e = sfg_setup + sfg_run from host arrays."""
    import torch
    from seisfem_b200.api import Context, Plan
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    dev = 0
    torch.cuda.set_device(dev)
    prob = workload(args.workload)
    N, steps = prob.mesh.node_num, prob.step - 2
    ctx = Context(dev)
    ctx.setup(prob)
    stream = torch.cuda.Stream(dev)
    sh = stream.cuda_stream
    plan = Plan(ctx, prob, precision="fp64cm", snap_every=0)
    for _ in range(args.warmup):
        plan.launch(0, sh)
    torch.cuda.synchronize(dev)
    plan.finish(0, stream=sh)
    cpath = os.path.join(tempfile.gettempdir(), "sfg_clocks_cm.csv")
    cproc, cf = clocks_start(cpath)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.launch(0, sh)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = clocks_stop(cproc, cf, cpath, dev)
    ms = e0.elapsed_time(e1) / args.steps
    res = plan.finish(0, stream=sh)
    st = ctx.stats()
    iters = int(st["cm_iterations"])
    launches = plan.launches
    plan.close()
    b_run = consistent_bytes(N, st["union_nnz"], steps, iters)
    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = b_run / (ms * 1e-3) / 1e9
    times = []
    for _ in range(2):
        t0 = time.perf_counter()
        c2 = Context(dev)
        c2.setup(prob)
        c2.run(prob, precision="fp64cm", snap_every=200)
        times.append(time.perf_counter() - t0)
        c2.close()
    m, md = prob.mesh, prob.model
    h2d = sum(a.nbytes for a in (m.element_node, m.x, m.y, md.rho, md.vp, md.vs, md.c))
    ns = ctx.L.sfg_snapshot_rows(prob.step, 200)
    d2h = 2 * 8 * steps * len(prob.rec_node) + 2 * 8 * ns * N
    dof_steps = 2 * N * steps
    line = {"metric": METRIC, "value": dof_steps / (ms * 1e-3), "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": prob.name, "element": m.type_name, "nodes": N, "dof": prob.dof,
                       "time_steps": steps, "dt": prob.dt, "solver": "consistent mass (pardiso / mgmres branch)",
                       "cg_iterations_per_time_step": iters / steps, "union_nnz": st["union_nnz"],
                       "l2": "CG vectors (6 x 14 doubles per node) + matrix: fits L2 at this size"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "algorithmic_bytes_per_run": b_run,
                         "note": "whole run (step kernels + CG iterations) over its CUDA-event time"},
            "e2e": {"value": dof_steps / float(min(times)), "unit": METRIC, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "cpu_baseline": None if args.no_cpu_baseline else cpu_baseline(args.workload, solver="mgmres", nsteps=4),
            "clocks": clocks, "gpu_launches": launches * args.steps, "energy_status": int(res["status"])}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_surrogate(args):
    """Config 5: FEM-generated training shots (Q4 128x128, GRF models, a
    source drawn along the surface, 64 receivers x 1000 samples), FNO training
    on the GPU, then held-out shots judged by the FEM: surrogate shots/s at
    its measured relative L2 error, beside the FEM's shots/s."""
    import torch
    from seisfem_b200.surrogate import (Surrogate, from_reduced_time, generate, moveout_samples, rel_l2,
                                        to_reduced_time)
    from seisfem_b200.surrogate import hybrid as hybrid_run
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ntr, nte = args.train_shots, args.test_shots
    t0 = time.perf_counter()
    xtr, ytr, fem_tr = generate(range(5000, 5000 + ntr))
    t_gen = time.perf_counter() - t0
    xte, yte, fem_te = generate(range(9000, 9000 + nte))
    # reduced time: the network learns the traces advanced by their moveout
    # at args.moveout_speed (exactly undone on its predictions)
    sh_tr = sh_te = None
    if args.moveout_speed > 0:
        sh_tr = moveout_samples(range(5000, 5000 + ntr), speed=args.moveout_speed)
        sh_te = moveout_samples(range(9000, 9000 + nte), speed=args.moveout_speed)
        ytr = to_reduced_time(ytr, sh_tr)
    sg = Surrogate(B=16, seed=0)
    K = sg.net.K
    # one timed training step for the tensor-core rate (FLOPs counted per GEMM)
    f0 = K.flops
    t1 = time.perf_counter()
    hist = sg.fit(xtr, ytr, epochs=args.epochs, lr=args.lr)
    torch.cuda.synchronize(dev)
    t_train = time.perf_counter() - t1
    train_flops = K.flops - f0
    steps = args.epochs * (ntr // 16)
    # inference: warm-up, then K timed passes over the held-out set (CUDA events;
    # inputs already on the device: value; with host copies: e2e)
    B = args.infer_batch
    inet = sg.inference_net(B)
    K = inet.K
    xb = torch.tensor(xte[:B]).to(dev).to(torch.bfloat16).contiguous()
    for _ in range(max(3, args.warmup)):
        inet.forward(xb, keep_pre=False)
    torch.cuda.synchronize(dev)
    f1 = K.flops
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(1, args.steps) * max(1, nte // B)
    e0.record()
    for _ in range(reps):
        inet.forward(xb, keep_pre=False)
    e1.record()
    torch.cuda.synchronize(dev)
    fwd_ms = e0.elapsed_time(e1) / reps
    fwd_flops = (K.flops - f1) / reps
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    pred = sg.predict(xte, batch=B)
    if sh_te is not None:
        pred = from_reduced_time(pred, sh_te)
    torch.cuda.synchronize(dev)
    t_e2e = time.perf_counter() - t2
    err = rel_l2(pred, yte)
    fallback = err > 1e-2
    # the hybrid at other bounds: every shot runs the surrogate; shots whose
    # error passes the bound run the FEM too (an exact error oracle: the
    # fraction is the best case of any error estimate)
    hybrid_by_bound = []
    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    peak = peaks.get("bf16_tflops", 1590.0)
    # batched FEM, one model per shot: set-up, per-batch coefficient streams,
    # loop and copies, the process's one-time CUDA start-up excluded
    fem_rate = 1.0 / float(fem_tr[-1])
    sur_rate = B / (fwd_ms * 1e-3)
    # hybrid pipeline: every shot runs the surrogate; shots over the bound run the FEM too
    hybrid = hybrid_run(err, 1e-2, 1.0 / sur_rate, 1.0 / fem_rate)["shots_per_s"]
    for bound in (1e-2, 0.05, 0.1, 0.2, 0.3, 0.4, 0.5):
        h = hybrid_run(err, bound, 1.0 / sur_rate, 1.0 / fem_rate)
        hybrid_by_bound.append({"bound": bound, "fallback_fraction": h["fallback_fraction"],
                                "hybrid_shots_per_s": h["shots_per_s"]})
    met = [h["bound"] for h in hybrid_by_bound if h["fallback_fraction"] <= 0.1]
    line = {"metric": "surrogate shots/s", "value": sur_rate, "unit": "shots/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": fwd_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": "config5_q4_128_fno", "train_shots": ntr, "test_shots": nte,
                       "grid": [128, 64], "samples": 1000, "width": 64, "modes": 16, "layers": 4,
                       "train_batch": sg.B, "inference_batch": B, "epochs": args.epochs,
                       "reduced_time_speed": args.moveout_speed if args.moveout_speed > 0 else None},
            "rel_l2": {"mean": float(err.mean()), "median": float(np.median(err)),
                       "p10": float(np.percentile(err, 10)), "p90": float(np.percentile(err, 90))},
            "fallback_fraction": float(fallback.mean()), "fallback_bound": 1e-2,
            "fem_shots_per_s": fem_rate, "hybrid_shots_per_s": hybrid,
            "hybrid_by_bound": hybrid_by_bound,
            "bound_met_by_90_percent": met[0] if met else None,
            "e2e": {"value": nte / t_e2e, "unit": "shots/s",
                    "h2d_bytes_per_step": int(xte[:B].size * 2), "d2h_bytes_per_step": int(B * 2 * 64 * 1000 * 4)},
            "roofline": {"bound": "tensor", "achieved": fwd_flops / (fwd_ms * 1e-3) / 1e12, "peak": peak,
                         "unit": "TFLOP/s", "frac": fwd_flops / (fwd_ms * 1e-3) / 1e12 / peak, "traffic": None,
                         "flops_per_forward": fwd_flops},
            "train": {"seconds": t_train, "steps": steps, "ms_per_step": t_train / steps * 1e3,
                      "tflops": train_flops / t_train / 1e12, "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1]},
            "fem_generation_seconds": t_gen,
            "gpu_launches": sg.net.K.launches + (inet.K.launches if inet is not sg.net else 0)}
    print(json.dumps(line), flush=True)
    return 0


def run_group(args):
    """Config 3b: independent Q4 meshes of uneven sizes, each with its own
    autotuned launch shapes, advanced by one CUDA-graph launch (sfg_group:
    the plans' graphs side by side); the multi-mesh kernels (one class-A and
    one class-Z launch per time step for all meshes) and the same plans
    launched one after another are the comparisons."""
    import torch
    from seisfem_b200.api import Context, Group, Plan
    dev = 0
    torch.cuda.set_device(dev)
    probs = P.config_3b()
    stream = torch.cuda.Stream(dev)
    sh = stream.cuda_stream
    ctxs, plans = [], []
    for p in probs:
        c = Context(dev)
        c.setup(p)
        ctxs.append(c)
        plans.append(Plan(c, p, precision=args.precision, snap_every=0))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def time_group(g):
        for _ in range(args.warmup):
            g.launch(sh)
        torch.cuda.synchronize(dev)
        for pl in plans:
            pl.finish(0, stream=sh)
        e0.record(stream)
        for _ in range(args.steps):
            g.launch(sh)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / args.steps

    # the multi-mesh kernels (the comparison), then the group's default: the
    # plans' own graphs side by side
    os.environ["SFG_GROUP_FUSED"] = "1"
    fused = Group(plans)
    del os.environ["SFG_GROUP_FUSED"]
    ms_fused = time_group(fused)
    fused_launches = fused.launches
    fused_mode = fused.fused
    fused.close()
    grp = Group(plans)
    ms = time_group(grp)
    e0.record(stream)
    for pl in plans:
        pl.launch(0, sh)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_seq = e0.elapsed_time(e1)
    dof_steps = sum(2 * p.mesh.node_num * (p.step - 2) for p in probs)
    b_step = sum(step_bytes(c, p, 1) for c, p in zip(ctxs, probs))
    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    steps = probs[0].step - 2
    achieved = b_step * steps / (ms * 1e-3) / 1e9
    shapes = [launch_shape(c.stats()["rows_per_block"], 1) for c in ctxs]
    line = {"metric": METRIC, "value": dof_steps / (ms * 1e-3), "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "config3b_16_q4_meshes", "sizes": [int(round(p.mesh.node_num ** 0.5)) - 1
                                                                      for p in probs],
                       "nodes_total": sum(p.mesh.node_num for p in probs), "time_steps": steps,
                       "precision": args.precision, "shots_per_mesh": 1,
                       "l2": "per-step working set of all meshes > 126 MB L2"},
            "group_mode": "multi-mesh kernels (2 launches per time step)" if grp.fused else
                          "the plans' graphs as child graphs, side by side",
            "group_launch_shapes": grp.shapes,
            "launches_per_time_step": grp.launches / steps,
            "sequential_ms": ms_seq, "group_over_sequential": ms_seq / ms,
            "multi_mesh_kernels_ms": ms_fused if fused_mode else None,
            "multi_mesh_kernels_launches_per_time_step": fused_launches / steps if fused_mode else None,
            "group_over_multi_mesh_kernels": ms_fused / ms if fused_mode else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "algorithmic_bytes_per_step": b_step},
            "launch_shapes": shapes, "gpu_launches": grp.launches * args.steps, "e2e": None, "cpu_baseline": None}
    print(json.dumps(line), flush=True)
    grp.close()
    for pl in plans:
        pl.close()
    for c in ctxs:
        c.close()
    return 0


def run_gemm_engines(args):
    """The surrogate's GEMM descriptors timed on both engines of
    sfg_fno_gemm (mma.sync tiles, tcgen05 with TMEM accumulators)."""
    import torch
    from seisfem_b200.surrogate import Kernels
    K = Kernels()
    dev = torch.device("cuda", 0)
    WT, Hp, Cc = 64000, 128, 64
    cases = [("head 1: M=64000 N=128 K=64 x16, A m-contiguous", WT, Hp, Cc, (16, 1), (Cc * WT, 0, 1, WT),
              (0, 0, Hp, 1), (WT * Hp, 0, Hp, 1), 16 * Cc * WT, Cc * Hp, 16 * WT * Hp, torch.bfloat16),
             ("head 1, A k-contiguous", WT, Hp, Cc, (16, 1), (Cc * WT, 0, Cc, 1), (0, 0, Hp, 1), (WT * Hp, 0, Hp, 1),
              16 * Cc * WT, Cc * Hp, 16 * WT * Hp, torch.bfloat16),
             ("8192 x 8192 x 1024, FP32 out", 8192, 8192, 1024, (1, 1), (0, 0, 1024, 1), (0, 0, 1, 1024),
              (0, 0, 8192, 1), 8192 * 1024, 8192 * 1024, 8192 * 8192, torch.float32),
             ("W-DFT: M=131072 N=32 K=64", 131072, 32, 64, (1, 1), (0, 0, 64, 1), (0, 0, 32, 1), (0, 0, 32, 1),
              131072 * 64, 64 * 32, 131072 * 32, torch.bfloat16),
             ("time map: M=64 N=1000 K=128 x1024", 64, 1000, 128, (1024, 1), (128 * 64, 0, 1, 64), (0, 0, 1000, 1),
              (64 * 1000, 0, 1000, 1), 1024 * 128 * 64, 128 * 1000, 1024 * 64 * 1000, torch.bfloat16)]
    out = []
    # the head's first GEMM as the network runs it: bias, stored
    # pre-activation and GELU in the epilogue
    hpre = torch.empty(16 * WT * Hp, device=dev, dtype=torch.bfloat16)
    hbias = torch.randn(Hp, device=dev)
    cases.insert(1, ("head 1 + bias, pre, GELU epilogue", WT, Hp, Cc, (16, 1), (Cc * WT, 0, 1, WT), (0, 0, Hp, 1),
                     (WT * Hp, 0, Hp, 1), 16 * Cc * WT, Cc * Hp, 16 * WT * Hp, torch.bfloat16))
    for name, M, N, Kd, batch, a, b, c, asz, bsz, csz, cdt in cases:
        epi = dict(bias=hbias, pre=hpre, gelu=True) if "epilogue" in name else {}
        A = torch.randn(asz, device=dev).to(torch.bfloat16)
        B = torch.randn(bsz, device=dev).to(torch.bfloat16)
        C = torch.empty(csz, device=dev, dtype=cdt)
        row = {"gemm": name, "flops": 2 * M * N * Kd * batch[0] * batch[1]}
        for eng, key in ((1, "mma_sync_us"), (3, "tcgen05_cp_async_us"), (4, "tcgen05_tma_us"),
                         (2, "tcgen05_tma_persistent_us")):
            for _ in range(max(3, args.warmup)):
                K.gemm(A, B, C, M, N, Kd, a=a, b=b, c=c, batch=batch, engine=eng, **epi)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(10):
                K.gemm(A, B, C, M, N, Kd, a=a, b=b, c=c, batch=batch, engine=eng, **epi)
            e1.record()
            torch.cuda.synchronize(dev)
            row[key] = e0.elapsed_time(e1) / 10 * 1e3
        out.append(row)
        print(json.dumps(row), flush=True)
    # the whole network (config-5 sizes, 16 shots): forward, and a training
    # step (forward, loss, backward, Adam), with mma.sync throughout against
    # the automatic per-GEMM choice
    from seisfem_b200.surrogate import FNO, init_params
    Bn, D, W, T = 16, 128, 64, 1000
    net = FNO(init_params(64, D, T, Hp, seed=1), Bn, D, W, T, dev)
    x = torch.randn((Bn, 4, D, W), device=dev).to(torch.bfloat16)
    tgt = torch.randn((Bn, 2, W, T), device=dev).to(torch.bfloat16)
    row = {"network": "FNO width 64, 16 shots, 128 x 64 grid, 1000 samples"}
    for eng, key in ((1, "mma_sync"), (0, "auto")):
        net.K.engine = eng
        for nm, fn in (("forward", lambda: net.forward(x, keep_pre=False)),
                       ("train_step", lambda: net.train_step(x, tgt, 1e-4))):
            for _ in range(max(3, args.warmup)):
                fn()
            torch.cuda.synchronize(dev)
            f0 = net.K.flops
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(5):
                fn()
            e1.record()
            torch.cuda.synchronize(dev)
            row[f"{nm}_{key}_ms"] = e0.elapsed_time(e1) / 5
            row[f"{nm}_gemm_flops"] = (net.K.flops - f0) // 5
    print(json.dumps(row), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--precision", default="fp32k", choices=["fp32k", "fp32", "fp64", "plain"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the config-3a batched-vs-plain section of the default workload's line")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the FP64 run that the rel_l2 field compares the timed run's outputs with")
    ap.add_argument("--compare-plain", action="store_true",
                    help="also time the unfused path (one SpMV launch per product) on one shot")
    ap.add_argument("--train-shots", type=int, default=4096)
    ap.add_argument("--test-shots", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--infer-batch", type=int, default=64, help="surrogate shots per inference pass")
    ap.add_argument("--moveout-speed", type=float, default=0.0,
                    help="surrogate: train on traces advanced by their moveout at this speed (m/s); 0 = raw time")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference" and args.workload in ACOUSTIC_WORKLOADS:
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        c = P.acoustic_grf(**ACOUSTIC_WORKLOADS[args.workload])
        cpu = acoustic_reference(c, nsteps=args.warmup + args.steps)
        v = cpu["value"]
        print(json.dumps({"impl": "reference", "metric": "node-steps/s", "value": v, "unit": "node-steps/s",
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 / v * c.mesh.node_num, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": {"workload": c.name, "nodes": c.mesh.node_num,
                                     "time_steps_per_bench_step": 1},
                          "cpu_baseline": cpu,
                          "e2e": {"value": v, "unit": "node-steps/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload in ACOUSTIC_WORKLOADS:
        return run_acoustic(args)
    if args.workload == "q4_200_consistent":
        return run_consistent(args)
    if args.workload == "surrogate_q4_128":
        return run_surrogate(args)
    if args.workload == "q4_16meshes":
        return run_group(args)
    if args.workload == "fno_gemm_engines":
        return run_gemm_engines(args)

    import torch
    import torch.distributed as dist
    from seisfem_b200.api import Context, Plan

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = local
    torch.cuda.set_device(dev)
    from seisfem_b200.shots import gather_seismograms_device, shard_problem
    # the job's shot list (one shot per rank for one-source workloads),
    # sharded over the ranks; each rank advances its block with no
    # communication inside the time loop
    prob_all = workload(args.workload, world)
    prob = shard_problem(prob_all, rank, world)
    S = len(prob.src_node)
    S_all = len(prob_all.src_node)
    ctx = Context(dev)
    ctx.setup(prob)
    st = ctx.stats()
    # a dedicated (non-default) stream: the plan's graph and the timing events
    # are queued on the same stream
    stream = torch.cuda.Stream(dev)
    plan = Plan(ctx, prob, precision=args.precision, snap_every=200)
    sh = stream.cuda_stream
    assert sh != 0

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        plan.launch(0, sh)
    torch.cuda.synchronize(dev)
    plan.finish(0, stream=sh)      # energy bound check of the warm-up result

    clk_path = os.path.join(tempfile.gettempdir(), f"sfg_clocks_{rank}.csv")
    proc, fh = clocks_start(clk_path)
    barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.launch(0, sh)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clocks = clocks_stop(proc, fh, clk_path, dev)
    ms = e0.elapsed_time(e1)
    res = plan.finish(0, stream=sh)
    launches = plan.launches * args.steps
    st = ctx.stats()
    plan.close()
    ms_t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{dev}")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    dof_steps_rank = 2 * prob.mesh.node_num * S * (prob.step - 2)
    dof_steps_job = 2 * prob.mesh.node_num * S_all * (prob.step - 2)
    value = dof_steps_job * args.steps / (ms_max / 1e3)

    # the job's seismograms, collected once after the loop: this rank's block
    # copied device to device, then one all_gather over NCCL (outside the
    # timed region; there is no collective inside the time loop)
    gathered = None
    if world > 1:
        rows_, R_ = prob.step - 2, len(prob.rec_node)
        su = torch.empty((S, rows_, R_), dtype=torch.float64, device=f"cuda:{dev}")
        sw = torch.empty_like(su)
        plan_g = Plan(ctx, prob, precision=args.precision, snap_every=0)
        plan_g.launch(0, sh)
        plan_g.finish_device(0, su.data_ptr(), sw.data_ptr(), sh)
        plan_g.close()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        full_u = gather_seismograms_device(su, S_all, rank, world)
        full_w = gather_seismograms_device(sw, S_all, rank, world)
        torch.cuda.synchronize(dev)
        gathered = {"shots": S_all, "bytes": 2 * full_u.numel() * 8, "ms": (time.perf_counter() - t0) * 1e3,
                    "how": "all_gather_into_tensor of device tensors (NCCL)",
                    "finite": bool(torch.isfinite(full_u).all() and torch.isfinite(full_w).all())}

    # roofline: the fused step kernel alone (a plan without snapshot copies),
    # average launch time = loop time / time steps, on the launching stream
    plan2 = Plan(ctx, prob, precision=args.precision, snap_every=0)
    for _ in range(2):
        plan2.launch(0, sh)
    torch.cuda.synchronize(dev)
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(1, args.steps)
    k0.record(stream)
    for _ in range(reps):
        plan2.launch(0, sh)
    k1.record(stream)
    torch.cuda.synchronize(dev)
    kms = k0.elapsed_time(k1) / (reps * (prob.step - 2))
    plan2.close()
    b_step = step_bytes(ctx, prob, S)
    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = b_step / (kms * 1e-3) / 1e9
    traffic = None
    if os.path.exists(TRAFFIC_FILE):
        traffic = read_traffic(TRAFFIC_FILE, f"{args.workload}:{args.precision}")
    b_ref = reference_layout_bytes(ctx, prob, S)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": "stepA/stepZ fused step (SpMV + RHS + lumped solve + Newmark), both classes",
                "algorithmic_bytes_per_launch": b_step, "avg_launch_us": round(kms * 1e3, 3),
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback",
                "reference_layout_bytes_per_launch": b_ref,
                "reference_layout_frac": round(b_ref / (kms * 1e-3) / 1e9 / peak, 4)}

    # e2e: public C-ABI call with host buffers (GPU assembly + run + outputs)
    e2e = None
    if not args.no_e2e:
        m, md = prob.mesh, prob.model
        h2d = sum(a.nbytes for a in (m.element_node, m.x, m.y, md.rho, md.vp, md.vs, md.c)) + 8 * S + 4 * len(prob.rec_node)
        ns = ctx.L.sfg_snapshot_rows(prob.step, 200)
        d2h = 2 * 8 * S * (prob.step - 2) * len(prob.rec_node) + 2 * 8 * S * ns * m.node_num
        # two untimed calls, then the median of seven: single calls on a
        # shared host vary by up to ~1 s (context creation, set-up)
        times = []
        for k in range(2 + 7):
            barrier()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            c2 = Context(dev)
            c2.setup(prob)
            c2.run(prob, precision=args.precision, snap_every=200)
            torch.cuda.synchronize(dev)
            times.append(time.perf_counter() - t0)
            c2.close()
        t_e2e = torch.tensor([statistics.median(times[2:])], dtype=torch.float64, device=f"cuda:{dev}")
        if world > 1:
            dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
        e2e = {"value": dof_steps_job / float(t_e2e.item()), "unit": METRIC,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "seconds_per_step": float(t_e2e.item()),
               "seconds_timed_calls": [round(t, 4) for t in times[2:]],
               "note": "one elastic_wave()-equivalent call per step: sfg_setup (GPU assembly from host arrays) + "
                       "sfg_run (loop, seismograms and 200-step snapshots copied back); median of 7 calls after 2"}

    plain = None
    if args.compare_plain:
        one = np.ascontiguousarray(prob.src_node[:1])
        pp = Plan(ctx, prob, precision="plain", snap_every=0, src_node=one)
        pp.launch(0, sh)
        torch.cuda.synchronize(dev)
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        pp.launch(0, sh)
        p1.record(stream)
        torch.cuda.synchronize(dev)
        pms = p0.elapsed_time(p1)
        per_shot_plain = 2 * prob.mesh.node_num * (prob.step - 2) / (pms / 1e3)
        per_shot_fused = value / (world * S)
        plain = {"plain_single_shot_dof_steps_per_s": per_shot_plain, "plain_ms_per_shot": pms,
                 "plain_launches_per_time_step": pp.launches / (prob.step - 2),
                 "fused_per_shot_dof_steps_per_s": per_shot_fused,
                 "ratio_batched_over_plain_per_shot_cost": value / (world * per_shot_plain)}
        pp.close()

    parity = None
    if not args.no_parity and args.precision != "fp64":
        parity = fused_parity(ctx, prob, res)

    batched = None
    if world == 1 and args.workload == DEFAULT_WORKLOAD and not args.no_batched:
        batched = batched_section(dev, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.workload)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision != "fp64" else "f64",
                "data": "synthetic",
                "config": bench_config(prob_all, S_all // world if S_all % world == 0 else S_all / world, world),
                "run": {"precision": args.precision, "union_nnz": st["union_nnz"],
                        "setup_ms": round(st["setup_ms"], 1), "repo_libraries_loaded": mapped_repo_libraries()},
                "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks,
                "gpu_launches": launches,
                "launch_shape": launch_shape(st["rows_per_block"], S),
                "vs_plain_path": plain,
                "rel_l2": parity,
                "batched": batched,
                "gathered_seismograms": gathered,
                "energy_status": int(res["status"])}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    ctx.close()
    return 0


def rel_l2(a, b) -> float:
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


REFERENCE_FIXTURES = {"config1_q4_200": "config1", "config2_q9_400": "config2"}


def fused_parity(ctx, prob, res, shots=(0, -1)) -> dict:
    """Relative L2 errors (||a - b|| / ||b|| over each whole output array) of
    the timed run's seismograms and 200-step snapshots: against the FP64 GPU
    path (the reference's operation order) run once here on the same inputs,
    outside the timed region, and, where a committed fixture of the
    reference's own FP64 run of this workload exists, against its values (a
    subset: every few receivers, snapshots on a coarse node grid).  Batches
    compare their first and last shot."""
    S = len(prob.src_node)
    pick = sorted({s % S for s in shots})
    keys = [k for k in ("seis_u", "seis_w", "snap_u", "snap_w") if k in res]
    t0 = time.perf_counter()
    out = {"bound": 1e-4, "against": "FP64 GPU path, same inputs, every receiver and snapshot node",
           "shots_compared": pick}
    ref = {k: [] for k in keys}
    for s in pick:
        r = ctx.run(prob, precision="fp64", snap_every=200 if "snap_u" in res else 0,
                    src_node=prob.src_node[[s]], want_snapshots="snap_u" in res)
        for k in keys:
            ref[k].append(r[k][0])
    for k in keys:
        out[k] = max(rel_l2(res[k][s], ref[k][i]) for i, s in enumerate(pick))
    out["max"] = max(out[k] for k in keys)
    out["fp64_seconds"] = round(time.perf_counter() - t0, 2)
    name = REFERENCE_FIXTURES.get(prob.name)
    path = os.path.join(ROOT, "tests", "golden", f"{name}_reference.npz") if name else None
    if path and os.path.exists(path) and S == 1:
        f = np.load(path)
        rec, nodes = f["rec"], f["nodes"]
        sub = {"seis_u": res["seis_u"][0][:, rec], "seis_w": res["seis_w"][0][:, rec]}
        if "snap_u" in res:
            sub["snap_u"], sub["snap_w"] = res["snap_u"][0][:, nodes], res["snap_w"][0][:, nodes]
        fx = {k: rel_l2(v, f[k]) for k, v in sub.items()}
        fx64 = {k: rel_l2(ref[k][0][:, rec] if k.startswith("seis") else ref[k][0][:, nodes], f[k]) for k in sub}
        out["vs_reference_run"] = {
            "fixture": os.path.relpath(path, ROOT),
            "what": f"the reference's own FP64 elastic_wave() run of this workload: receivers every "
                    f"{int(rec[1] - rec[0])}, snapshot nodes on every {int(nodes[1] - nodes[0])}th grid line",
            "fp32": fx, "fp64_gpu": fx64, "max": max(fx.values())}
    return out


def batched_section(dev: int, stream, steps: int = 3, warmup: int = 3) -> dict:
    """The metric's own comparison on config 3a (Q4 400x400 GRF, 64 shots,
    2000 time steps): the 64-shot batch advanced as one SpMM-shaped fused
    step per time step, against the plain single-shot FP32 path (one
    csr_matvec launch per product, as elastic_wave.c structures the step) on
    one of its shots; DOF-steps/s, the fused kernels' roofline, and the
    batch's first and last shot against FP64 single-shot runs."""
    import torch
    from seisfem_b200.api import Context, Plan
    prob = workload("q4_400_grf_64shots")
    S, N, T = len(prob.src_node), prob.mesh.node_num, prob.step - 2
    sh = stream.cuda_stream
    ctx = Context(dev)
    ctx.setup(prob)
    plan = Plan(ctx, prob, precision="fp32k", snap_every=0)
    shape_code = ctx.stats()["rows_per_block"]   # the batch plan's pick (later plans overwrite the stats)
    for _ in range(warmup):
        plan.launch(0, sh)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        plan.launch(0, sh)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    res = plan.finish(0, stream=sh)
    launches = plan.launches
    plan.close()
    value = 2 * N * S * T / (ms * 1e-3)
    b_step = step_bytes(ctx, prob, S)
    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = b_step * T / (ms * 1e-3) / 1e9
    # the plain single-shot FP32 path on the batch's first shot
    pp = Plan(ctx, prob, precision="plain", snap_every=0, src_node=prob.src_node[:1])
    pp.launch(0, sh)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    pp.launch(0, sh)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    pms = e0.elapsed_time(e1)
    plain_rate = 2 * N * T / (pms * 1e-3)
    plain_launches = pp.launches / T
    pp.close()
    parity = fused_parity(ctx, prob, res)
    st = ctx.stats()
    ctx.close()
    return {"config": {"workload": prob.name, "element": "Q4", "nodes": N, "shots": S, "time_steps": T,
                       "precision": "fp32k", "union_nnz": st["union_nnz"],
                       "l2": "per-step working set > 126 MB L2; no flush needed"},
            "value": value, "unit": METRIC, "ms_per_run": ms, "runs_timed": steps, "warmup": warmup,
            "gpu_launches_per_run": launches,
            "launch_shape": launch_shape(shape_code, S),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "algorithmic_bytes_per_launch": b_step,
                         "avg_step_us": round(ms * 1e3 / T, 3),
                         "kernel": "stepA/stepZ batched fused step, 64 shots innermost",
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks
                         else "fallback"},
            "vs_plain_path": {"plain_single_shot_dof_steps_per_s": plain_rate, "plain_ms_per_shot": pms,
                              "plain_launches_per_time_step": plain_launches,
                              "batched_per_shot_dof_steps_per_s": value / S,
                              "ratio_batched_over_plain_per_shot_cost": value / plain_rate},
            "rel_l2": parity, "energy_status": int(res["status"])}


def launch_shape(code, S):
    """The autotuner's pick for the class-A / class-Z kernels."""
    if S == 1:
        return {"variant_A": code // 16, "variant_Z": code % 16}
    a, z = code // 256, code % 256
    return {"A": {"shots_per_lane": (a >> 4) & 15, "warps_per_block": a & 15, "staged_gathers": bool(a & 0x100)},
            "Z": {"shots_per_lane": z >> 4, "warps_per_block": z & 15}}


def read_traffic(path, key):
    """DRAM bytes per time step (dram__bytes_read.sum + dram__bytes_write.sum of
    the step's kernels) from the ncu summary table: lines `key bytes ...`."""
    for line in open(path):
        f = line.split()
        if len(f) >= 2 and f[0] == key:
            return int(f[1])
    return None


def reference_layout_bytes(ctx, prob, S) -> int:
    """Bytes per step of the unreduced layout: every union entry with its
    column and all 7 FP32 values, 64 state floats per node and shot (26
    fields, 6 compensations, read and written) and 11 coefficient streams
    per node: Z_u (4 + 7 w) + 4 (N + 1) + N w (64 S + 11), w = 4.  The
    kernels move fewer bytes (step_bytes); this is the work they replace."""
    N = prob.mesh.node_num
    Zu = int(ctx.stats()["union_nnz"])
    return Zu * (4 + 7 * 4) + 4 * (N + 1) + N * 4 * (64 * S + 11)


def step_bytes(ctx, prob, S) -> int:
    """Algorithmic bytes of one fused FP32 time step (all S shots), for the
    two-class layout.  Matrix: one shot streams SELL slots of column + M +
    K1..K4 (24 B per union entry) outside the M-PML and 32 B inside it (K5,
    K6 too), or, with the value dictionary, 8 B slots (column, tuple id) --
    4 B (halo position, tuple id) in a class run by the staged-gather tile
    kernels -- plus one density per row; batches read 32 B row records per
    entry.  State:
    rows outside the M-PML zone move their totals record (Gc 12 + Pa 4
    floats, read and written once), split-zone rows Gc + Gs + Ps (36 floats),
    per shot; per-node coefficients 5 floats (interior) or 12 (split zone).
    Gathers of neighbour records are counted once (their owner's read)."""
    p, j = ctx.union_pattern()
    L = np.diff(p).astype(np.int64)
    mp = ctx.mpml()
    pml = np.any(mp[:4].astype(np.float32) != 0, axis=0)
    zone = pml.copy()
    rows = np.repeat(np.arange(len(L)), L)
    zone[j[pml[rows]]] = True
    N = prob.mesh.node_num
    na = int((~zone).sum())
    na -= na % 32   # the last few class-A rows join class Z (a multiple of 32 stays in A)
    assert na == ctx.stats()["interior_rows"], (na, ctx.stats()["interior_rows"])
    if S > 1:
        mat = int(L.sum()) * 32 + 4 * (N + 1)
    elif ctx.stats()["value_tuples"] > 0:
        # slots of 8 B (column, tuple id), or 4 B (halo position, tuple id)
        # in a class that the staged-gather tile kernels (launch shape 6) run
        code = ctx.stats()["rows_per_block"]
        wa, wz = (4 if code // 16 == 6 else 8), (4 if code % 16 == 6 else 8)
        mat = int(L[~zone].sum()) * wa + int(L[zone].sum()) * wz + 4 * (N // 32 + 2) + 4 * N
    else:
        mat = int(L[pml].sum()) * 32 + int(L[~pml].sum()) * 24 + 4 * (N // 32 + 2)
    state = (na * (12 + 4) + (N - na) * (12 + 12 + 12)) * 4 * 2 * S
    coef = na * 5 * 4 + (N - na) * 12 * 4
    return int(mat + state + coef)


if __name__ == "__main__":
    sys.exit(main())
