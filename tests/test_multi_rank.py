"""Multi-rank shot sharding on CPU (gloo, world size 2): every rank advances
its own block of shots with no communication inside the time loop, and the
seismograms are collected once with one all_gather of tensors.  The ranks
run the same code as bench.py --gpus N (shots.run_sharded with a runner per
rank); here the runner is the CPU oracle, on GPUs it is api.device_runner
(a Plan on the rank's device) and the collective goes over NCCL."""
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


def _oracle_runner(sub):
    import torch
    from oracle import Oracle
    out = Oracle().run(sub, nthreads=1)
    return torch.from_numpy(out["seis_u"]), torch.from_numpy(out["seis_w"])


def _worker(rank, world, port, out_path, shots):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    import datetime
    import torch.distributed as dist
    from seisfem_b200.problem import small_problem
    from seisfem_b200.shots import gather_seismograms, run_sharded, shard_problem
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    p = small_problem("Q4", n=12, step=120, pml=2, seed=3, shots=shots)
    su, sw = run_sharded(p, rank, world, _oracle_runner)
    # the host-array gather agrees with the tensor gather
    host = gather_seismograms(_oracle_runner(shard_problem(p, rank, world))[0].numpy(), shots, rank, world)
    if rank == 0:
        assert np.array_equal(host, su.numpy())
        np.savez(out_path, seis_u=su.numpy(), seis_w=sw.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("shots", [5, 1])
def test_two_ranks_match_single_process(tmp_path, oracle, shots):
    """5 shots (3 + 2: uneven shards) and 1 shot (one rank has none)."""
    import torch.multiprocessing as mp
    from seisfem_b200.problem import small_problem
    out = str(tmp_path / "gathered.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out, shots), nprocs=2, join=True, start_method="spawn")
    gathered = np.load(out)
    ref = oracle.run(small_problem("Q4", n=12, step=120, pml=2, seed=3, shots=shots), nthreads=1)
    for k in ("seis_u", "seis_w"):
        assert gathered[k].shape == ref[k].shape
        assert np.array_equal(gathered[k], ref[k])


# ---------------------------------------------------------------- surrogate

FNO_SMALL = dict(B=2, C_=8, Hp=16, D=32, W=32, T=48)


def _fno_data(n=8, seed=6):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, 4, FNO_SMALL["D"], FNO_SMALL["W"])).astype(np.float32)
    y = rng.standard_normal((n, 2, FNO_SMALL["W"], FNO_SMALL["T"])).astype(np.float32)
    return x, y


def _fno_worker(rank, world, port, out_path):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "tests")]
    import datetime
    import torch.distributed as dist
    from fno_emulator import EmuKernels
    from seisfem_b200.surrogate import Surrogate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    x, y = _fno_data()
    sg = Surrogate(**FNO_SMALL, device="cpu", kernels=EmuKernels(), seed=1)
    hist = sg.fit(x, y, epochs=2, lr=1e-3, seed=3, group=dist.group.WORLD)
    if rank == 0:
        np.savez(out_path, hist=np.array(hist), **sg.net.params_numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_surrogate_data_parallel_matches_one_process(tmp_path):
    """Two gloo ranks, 2 shots each per step, gradients averaged by one
    all-reduce: the weights and losses of one process training on the same
    4-shot batches (the kernels emulated on the CPU)."""
    import sys
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from fno_emulator import EmuKernels
    from seisfem_b200.surrogate import Surrogate
    out = str(tmp_path / "dp.npz")
    mp.start_processes(_fno_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    dp = np.load(out)
    x, y = _fno_data()
    one = Surrogate(**{**FNO_SMALL, "B": 4}, device="cpu", kernels=EmuKernels(), seed=1)
    hist = one.fit(x, y, epochs=2, lr=1e-3, seed=3)
    assert np.allclose(dp["hist"], hist, rtol=1e-4)
    ref = one.net.params_numpy()
    for k, v in ref.items():
        d = np.linalg.norm(dp[k] - v) / max(np.linalg.norm(v), 1e-30)
        assert d < 1e-4, (k, d)
