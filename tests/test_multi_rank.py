"""Multi-rank shot sharding on CPU (gloo, world size 2): every rank advances
its own block of shots with no communication inside the time loop, and the
seismograms are gathered once on rank 0.  The per-rank compute here is the
CPU oracle; on GPUs it is the same code path with sfg_run per rank."""
import os
import socket

import numpy as np
import pytest

from seisfem_b200.shots import shard


def test_shard_covers_every_shot_once():
    for n in (1, 2, 7, 64, 65):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                s = shard(n, r, world)
                got += list(range(n))[s]
            assert got == list(range(n))
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    import datetime
    import torch.distributed as dist
    from oracle import Oracle
    from seisfem_b200.problem import small_problem
    from seisfem_b200.shots import gather_seismograms, shard as shard_
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    p = small_problem("Q4", n=12, step=120, pml=2, seed=3, shots=5)
    mine = shard_(len(p.src_node), rank, world)
    p.src_node = p.src_node[mine]
    local = Oracle().run(p, nthreads=1)["seis_u"]
    full = gather_seismograms(local, 5, rank, world)
    if rank == 0:
        np.save(out_path, full)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_match_single_process(tmp_path, oracle):
    import torch.multiprocessing as mp
    from seisfem_b200.problem import small_problem
    out = str(tmp_path / "gathered.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    gathered = np.load(out)
    ref = oracle.run(small_problem("Q4", n=12, step=120, pml=2, seed=3, shots=5), nthreads=1)["seis_u"]
    assert gathered.shape == ref.shape
    assert np.array_equal(gathered, ref)
