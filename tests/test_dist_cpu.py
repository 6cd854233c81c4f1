"""Sharded sweep across ranks: world_size-2 gloo processes on CPU.

Each rank takes its LPT share of a batch of ROMs, sweeps it with the CPU restatement (the
GPU kernels are not needed to test the partitioning), and rank 0 gathers everything and
compares with a single-process sweep; the step-time reduction is the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from staccato_b200 import dist as D


def test_partition_covers_every_item_once_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.uniform(1, 100, size=97))
    for world in (1, 2, 3, 8):
        parts = D.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-9
    with pytest.raises(ValueError):
        D.partition(costs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist

    from oracle import oracle as O
    from staccato_b200 import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    roms = W.batching_roms(count=6, n_lo=8, n_hi=24, F_lo=3, F_hi=6)
    parts = D.partition([D.rom_cost(r.n, r.r, r.F) for r in roms], world)
    mine = parts[rank]
    res = {}
    for i in mine:
        r = roms[i]
        X, _ = O.sweep(r.K, r.M, r.D, 0.0, r.rhs, r.omega)
        res[i] = X
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    t = D.max_over_ranks(float(rank + 1))
    if rank == 0:
        allres = {}
        for g in gathered:
            allres.update(g)
        np.savez(os.path.join(out_dir, "gathered.npz"), **{str(k): v for k, v in allres.items()},
                 tmax=np.array(t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_sharded_sweep(tmp_path):
    from oracle import oracle as O
    from staccato_b200 import workloads as W

    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    data = np.load(tmp_path / "gathered.npz")
    roms = W.batching_roms(count=6, n_lo=8, n_hi=24, F_lo=3, F_hi=6)
    assert float(data["tmax"]) == 2.0
    for i, r in enumerate(roms):
        X, _ = O.sweep(r.K, r.M, r.D, 0.0, r.rhs, r.omega)
        assert np.array_equal(data[str(i)], X)


def test_frequency_slices_cover_once_and_balance():
    from staccato_b200.dist import frequency_slice

    for n_freq in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            sl = [frequency_slice(n_freq, world, r) for r in range(world)]
            assert sl[0][0] == 0 and sl[-1][1] == n_freq
            assert all(sl[i][1] == sl[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in sl]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        frequency_slice(10, 2, 2)
