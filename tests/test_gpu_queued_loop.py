"""The time loop of large runs (sfg_run on meshes whose node count times the
batch's shot count reaches 2^18) is queued as 16 direct steps and then as
graphs of up to 256 steps that end after snapshot steps, two executable
graphs updated in place in turn; snapshot rows go to the caller on a copy
stream one chunk behind (an event per row, row 0 after the state reset).  A
plan (sfg_plan_*) captures the same loop as one graph and copies the rows at
the end.  The two give the same outputs bit for bit (snapshots every 25
steps, so that chunks start on both parities of the ping-pong state
buffers)."""
import numpy as np
import pytest

from seisfem_b200.problem import small_problem

pytestmark = pytest.mark.gpu

KEYS = ("seis_u", "seis_w", "snap_u", "snap_w")


def _run_both(prob, precision, spb):
    from seisfem_b200.api import Context, Plan
    ctx = Context(0)
    try:
        ctx.setup(prob)
        run = ctx.run(prob, precision=precision, shots_per_batch=spb, snap_every=25)
        plan = Plan(ctx, prob, precision=precision, snap_every=25, shots_per_batch=spb)
        plan.launch(0)
        one = plan.finish(0)
        launches = plan.launches
        plan.close()
        stats = ctx.stats()
    finally:
        ctx.close()
    return run, one, launches, stats


@pytest.mark.parametrize("precision", ["fp32k", "fp64"])
def test_one_shot_queued_loop_equals_one_graph(precision):
    prob = small_problem("Q4", n=512, step=122, pml=10, seed=3)
    assert prob.mesh.node_num >= 1 << 18           # sfg_run queues the loop in chunks
    run, one, launches, stats = _run_both(prob, precision, 1)
    assert run["status"] == 0 and one["status"] == 0
    for k in KEYS:
        assert np.array_equal(run[k], one[k]), k
    assert np.linalg.norm(one["snap_u"][0, -1]) > 0     # the wave reached the snapshots
    assert stats["kernel_launches"] == launches        # the chunks queue the plan's kernels


def test_batched_queued_loop_equals_one_graph():
    prob = small_problem("Q4", n=64, step=122, pml=6, shots=64, seed=11)
    assert prob.mesh.node_num * 64 >= 1 << 18
    run, one, launches, stats = _run_both(prob, "fp32k", 64)
    assert run["status"] == 0 and one["status"] == 0
    for k in KEYS:
        assert np.array_equal(run[k], one[k]), k
    assert stats["kernel_launches"] == launches


def test_two_batches_reuse_the_chunk_graphs():
    """96 shots in batches of 64: the second (ragged) batch's chunks update
    the graphs the first batch's chunks left in the plan."""
    from seisfem_b200.api import Context, Plan
    prob = small_problem("Q4", n=64, step=122, pml=6, shots=96, seed=12)
    assert prob.mesh.node_num * 64 >= 1 << 18
    ctx = Context(0)
    try:
        ctx.setup(prob)
        run = ctx.run(prob, precision="fp32k", shots_per_batch=64, snap_every=25)
        plan = Plan(ctx, prob, precision="fp32k", snap_every=25, shots_per_batch=64)
        assert plan.batches == 2
        outs = []
        for b in range(2):
            plan.launch(b)
            outs.append(plan.finish(b))
        plan.close()
    finally:
        ctx.close()
    assert run["status"] == 0
    for k in KEYS:
        one = np.concatenate([outs[0][k][:64], outs[1][k][64:]])   # each batch at its shots' offset
        assert np.array_equal(run[k], one), k
