"""Config 4 (T6 mesh, sinusoidal free-surface topography, VTI) and config 3b
(uneven meshes in one CUDA-graph launch) at sizes the oracle finishes in
seconds."""
import copy

import numpy as np
import pytest

from conftest import rel_l2
from seisfem_b200.problem import config_3b, config_4

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4


def test_config4_small_fp32_matches_oracle(ctx, oracle):
    # 30 x 60 T6 elements with the same topography, medium and time step; 200
    # steps lie inside the window before the reference's T6 energy bound trips
    p = config_4(nx=30, ny=60, pml=5, step=202)
    ref = oracle.run(p)
    assert ref["status"] == 0
    ctx.setup(p)
    out = ctx.run(p, precision="fp32k")
    for k in ("seis_u", "seis_w", "snap_u", "snap_w"):
        assert rel_l2(out[k], ref[k]) < FP32_TOL, (k, rel_l2(out[k], ref[k]))
    # the free surface is not Dirichlet: surface receivers move
    assert np.abs(out["seis_u"]).max() > 0


def test_config4_t6_energy_bound_trips_like_the_reference(ctx, oracle):
    """The reference's lumped T6 scheme with its M-PML grows without bound
    (flat or sinusoidal top, isotropic or VTI, dt 0.1-0.4 ms); the oracle
    and both GPU precisions stop at the energy bound, the FP32 path within a
    few steps of the FP64 one."""
    p = config_4(nx=30, ny=60, pml=5, step=400)
    ref = oracle.run(p)
    assert ref["status"] == 1
    ctx.setup(p)
    o64 = ctx.run(p, precision="fp64", raise_on_blowup=False)
    o32 = ctx.run(p, precision="fp32k", raise_on_blowup=False)
    assert o64["status"] == 6 and o32["status"] == 6
    b64, b32 = o64["stats"]["blowup_step"], o32["stats"]["blowup_step"]
    assert 200 < b64 < 400 and abs(b32 - b64) <= 3, (b64, b32)


@pytest.mark.parametrize("mode", ["fused", "child_graphs"])
def test_group_launch_matches_separate_plans(oracle, mode, monkeypatch):
    """Uneven meshes in one graph launch -- one class-A and one class-Z
    kernel per time step for all meshes ("fused"), or the plans' own graphs
    side by side -- give each plan's own results bit for bit, on repeated
    launches."""
    from seisfem_b200.api import Context, Group, Plan
    if mode == "fused":
        monkeypatch.setenv("SFG_GROUP_FUSED", "1")
    else:
        monkeypatch.delenv("SFG_GROUP_FUSED", raising=False)
    probs = config_3b(count=3, lo=20, hi=50, step=202, pml=4)
    assert len({p.mesh.node_num for p in probs}) == 3
    ctxs = [Context(0) for _ in probs]
    for c, p in zip(ctxs, probs):
        c.setup(p)
    plans = [Plan(c, p, precision="fp32k", snap_every=200) for c, p in zip(ctxs, probs)]
    alone = []
    for pl in plans:
        pl.launch(0)
        alone.append(pl.finish(0))
    grp = Group(plans)
    assert grp.fused == (mode == "fused")
    steps = probs[0].step - 2
    if grp.fused:
        # two kernels per time step for all meshes, plus per mesh one
        # snapshot (step 199) and the last receiver row
        assert grp.launches == 2 * steps + 2 * len(plans), grp.launches
    else:
        assert grp.launches == sum(pl.launches for pl in plans)
    for _ in range(2):       # twice: every launch starts from the zero state
        grp.launch()
        for c in ctxs:
            c.L.sfg_sync(c.ptr)
        for pl, a, p in zip(plans, alone, probs):
            out = pl.finish(0)
            for k in ("seis_u", "seis_w", "snap_u", "snap_w"):
                assert np.array_equal(out[k], a[k]), k
    ref = oracle.run(probs[1])
    got = plans[1].finish(0)
    for k in ("seis_u", "seis_w"):
        assert rel_l2(got[k], ref[k]) < FP32_TOL, k
    grp.close()
    for pl in plans:
        pl.close()
    for c in ctxs:
        c.close()


def test_group_of_mixed_plans_composes_child_graphs():
    """A group with a batched plan cannot share the one-shot multi-mesh
    kernels: it falls back to the plans' own graphs, still bit for bit."""
    from seisfem_b200.api import Context, Group, Plan
    from seisfem_b200.problem import small_problem
    probs = [small_problem("Q4", n=24, step=122, pml=4, seed=2),
             small_problem("Q4", n=30, step=122, pml=4, seed=3, shots=32)]
    ctxs = [Context(0) for _ in probs]
    for c, p in zip(ctxs, probs):
        c.setup(p)
    plans = [Plan(c, p, precision="fp32k", snap_every=0, shots_per_batch=len(p.src_node)) for c, p in zip(ctxs, probs)]
    alone = []
    for pl in plans:
        pl.launch(0)
        alone.append(pl.finish(0))
    grp = Group(plans)
    assert not grp.fused
    grp.launch()
    for c in ctxs:
        c.L.sfg_sync(c.ptr)
    for pl, a in zip(plans, alone):
        out = pl.finish(0)
        for k in ("seis_u", "seis_w"):
            assert np.array_equal(out[k], a[k]), k
    grp.close()
    for pl in plans:
        pl.close()
    for c in ctxs:
        c.close()


def _models_case(shots, seed0=5000, **kw):
    from seisfem_b200.problem import config_5
    probs = [config_5(seed0 + k, **kw) for k in range(shots)]
    p = copy.copy(probs[0])
    p.src_node = np.concatenate([q.src_node for q in probs]).astype(np.int32)
    return p, probs


def test_one_model_per_shot_matches_separate_runs(oracle):
    """Batched shots with their own GRF models (config 5 recipe, smaller
    mesh) against each shot run alone in a context set up with its model,
    and two shots against the FP64 oracle."""
    from seisfem_b200.api import Context
    shots = 35                       # one full batch of 32 and a ragged one
    p, probs = _models_case(shots, n=40, samples=200, nrec=16, pml=6)
    ctx = Context(0)
    ctx.setup(probs[0])
    got = ctx.run_models(p, [q.model for q in probs], shots_per_batch=32, snap_every=200)
    for k in (0, 7, 33):
        c2 = Context(0)
        c2.setup(probs[k])
        one = c2.run(probs[k], precision="fp32k", snap_every=200)
        c2.close()
        for key in ("seis_u", "seis_w", "snap_u", "snap_w"):
            assert rel_l2(got[key][k], one[key][0]) < 1e-5, (k, key, rel_l2(got[key][k], one[key][0]))
    for k in (3, 34):
        ref = oracle.run(probs[k])
        for key in ("seis_u", "seis_w"):
            assert rel_l2(got[key][k], ref[key][0]) < FP32_TOL, (k, key)
    ctx.close()


def test_one_model_per_shot_same_model_equals_batched_run():
    from seisfem_b200.api import Context
    p, probs = _models_case(40, n=40, samples=150, nrec=16, pml=6)
    same = [probs[0].model] * 40
    ctx = Context(0)
    ctx.setup(probs[0])
    a = ctx.run_models(p, same, shots_per_batch=64)
    b = ctx.run(p, precision="fp32k", shots_per_batch=64, snap_every=0, want_snapshots=False)
    for key in ("seis_u", "seis_w"):
        assert rel_l2(a[key], b[key]) < 1e-6, key
    ctx.close()
