"""Shot-parallel host logic on CPU: partitioning and the cross-rank sums,
with torch.distributed over gloo, world size 2 (two local processes)."""
import os
import socket

import numpy as np
import pytest

from fwi3d_b200 import shots


def test_round_robin_partition_covers_every_shot_once():
    for n, world in ((64, 1), (64, 8), (7, 3), (2, 4)):
        parts = [shots.partition(n, world, r) for r in range(world)]
        allv = sorted(s for p in parts for s in p)
        assert allv == list(range(n))


def test_cost_partition_balances_load():
    rng = np.random.default_rng(0)
    costs = rng.integers(5000, 15000, 64).astype(float)
    parts = [shots.partition(64, 4, r, costs) for r in range(4)]
    assert sorted(s for p in parts for s in p) == list(range(64))
    loads = [costs[p].sum() for p in parts]
    assert max(loads) - min(loads) <= costs.max()
    # deterministic: every rank computes the same assignment
    assert parts == [shots.partition(64, 4, r, costs) for r in range(4)]


def test_bad_arguments():
    with pytest.raises(ValueError):
        shots.partition(4, 2, 2)
    with pytest.raises(ValueError):
        shots.partition(4, 2, 0, costs=[1.0, 2.0])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shots.partition(10, world, rank)
        # each rank "images" its own shots: shot s contributes s+1 everywhere
        img = torch.zeros(6, 5, 4)
        ill = torch.zeros(6, 5, 4)
        for s in mine:
            img += s + 1
            ill += 2 * (s + 1)
        shots.sum_across_ranks(img, ill)
        misfit = shots.misfit_across_ranks(sum(0.1 * (s + 1) for s in mine))
        q.put((rank, mine, float(img[0, 0, 0]), float(ill[5, 4, 3]), misfit))
    finally:
        dist.destroy_process_group()


def test_two_rank_image_and_misfit_sums():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert sorted(out[0][1] + out[1][1]) == list(range(10))
    want = sum(range(1, 11))
    for _, _, img, ill, misfit in out:
        assert img == want and ill == 2 * want
        assert abs(misfit - 0.1 * want) < 1e-12
