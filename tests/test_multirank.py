"""Multi-rank host logic on CPU: two gloo ranks (the GPU path runs the same
code with NCCL, one process per GPU, independent volumes per rank)."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, cells, out):
    import datetime

    import torch.distributed as dist

    from hpmc_b200 import multi

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        parts = multi.split_volumes(cells, world)
        mine = parts[rank]
        # a stand-in device time proportional to this rank's work
        t = float(sum(cells[i] for i in mine)) * 1e-9 + rank * 1e-6
        t_max = multi.max_over_ranks(t)
        n_all = multi.sum_over_ranks(len(mine))
        out.put((rank, mine, t, t_max, n_all))
    finally:
        dist.destroy_process_group()


def test_split_is_a_balanced_partition():
    from hpmc_b200 import datasets, multi

    rng = __import__("numpy").random.default_rng(3)
    cells = [int(e) ** 3 for e in rng.integers(32, 193, size=64)]
    for world in (1, 2, 4, 8):
        parts = multi.split_volumes(cells, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells)  # greedy longest-first bound
    assert multi.split_volumes(cells, 2) == multi.split_volumes(list(cells), 2)  # deterministic
    del datasets


def test_two_gloo_ranks_agree_on_split_and_max_time():
    import torch.multiprocessing as mp

    cells = [40 ** 3, 192 ** 3, 64 ** 3, 100 ** 3, 32 ** 3, 150 ** 3, 77 ** 3]
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, cells, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mine = [r[1] for r in res]
    assert sorted(mine[0] + mine[1]) == list(range(len(cells))) and not set(mine[0]) & set(mine[1])
    t_max = max(r[2] for r in res)
    assert all(abs(r[3] - t_max) < 1e-12 for r in res)  # every rank sees the same maximum
    assert all(r[4] == len(cells) for r in res)


def test_single_process_fallbacks():
    from hpmc_b200 import multi

    assert multi.max_over_ranks(1.5) == 1.5
    assert multi.sum_over_ranks(3) == 3.0
