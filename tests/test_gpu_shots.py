"""The per-rank runner of the multi-GPU shot path (api.device_runner, used
by shots.run_sharded and bench.py --gpus N) on one GPU: seismograms written
to device tensors match the host-buffer run of the same shots, for a
one-shot plan and for a batch with a ragged tail."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from seisfem_b200.problem import small_problem
from seisfem_b200.shots import run_sharded, shard_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shots", [1, 37])
def test_device_runner_matches_host_run(ctx, shots):
    from seisfem_b200.api import device_runner
    p = small_problem("Q4", n=30, step=152, pml=4, seed=9, shots=shots)
    ctx.setup(p)
    su, sw = run_sharded(p, 0, 1, device_runner(ctx))
    assert su.is_cuda and su.shape == (shots, p.step - 2, len(p.rec_node))
    host = ctx.run(p, precision="fp32k", want_snapshots=False)
    assert np.array_equal(su.cpu().numpy(), host["seis_u"])
    assert np.array_equal(sw.cpu().numpy(), host["seis_w"])


def test_device_runner_shards_cover_the_shot_list(ctx):
    """Each of three would-be ranks runs its shard; the blocks, stacked in
    rank order, are the whole shot list's seismograms."""
    from seisfem_b200.api import device_runner
    p = small_problem("Q4", n=24, step=102, pml=3, seed=4, shots=5)
    ctx.setup(p)
    run = device_runner(ctx)
    parts = [run(shard_problem(p, r, 3))[0] for r in range(3)]
    assert [t.shape[0] for t in parts] == [2, 2, 1]
    whole = run(p)[0]
    assert rel_l2(torch.cat(parts).cpu().numpy(), whole.cpu().numpy()) == 0.0
