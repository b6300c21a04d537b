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


class FakeContext:
    """Stands in for lib.Context on the CPU so that fwi.Fwi's shot partition
    and cross-rank sums can run under gloo: a shot's 'seismogram' is a fixed
    function of the shot and the velocity, and a shot's 'gradient' adds a
    shot-dependent pattern scaled by its residual.  Device pointers are the
    addresses of CPU tensors."""

    def __init__(self, w):
        self.nzz, self.nxx, self.nyy = w.nz + 2 * w.nb, w.nx + 2 * w.nb, w.ny + 2 * w.nb
        self.nb, self.nt = w.nb, w.nt
        shape = (self.nyy, self.nxx, self.nzz)
        self.img, self.ill = np.zeros(shape, np.float32), np.zeros(shape, np.float32)
        self.seeds = []

    @staticmethod
    def _view(ptr, n):
        import ctypes
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)), shape=(n,))

    def set_geometry(self, src, rec, first, count):
        self.count = np.full(len(src), len(rec)) if count is None else np.asarray(count)

    def shot_nrec(self, s):
        return int(self.count[s])

    def set_velocity(self, v):
        self.v = np.asarray(v, np.float64)

    def model_shots_dev(self, shots_, ptr):
        off = 0
        for s in shots_:
            n = self.shot_nrec(s) * self.nt
            i = np.arange(n)
            seis = np.sin(1e-3 * (s + 1) * i) * self.v.mean() / 1000.0 + np.cos(self.v.ravel()[s] * 1e-3 + i)
            self._view(ptr + 4 * off, n)[:] = seis.astype(np.float32)
            off += n

    def residual_dev(self, obs, cal, n, res):
        r = self._view(obs, n) - self._view(cal, n)
        self._view(res, n)[:] = r
        return float(np.sum(r.astype(np.float64) ** 2))

    def reset_accumulators(self):
        self.img[:] = 0
        self.ill[:] = 0

    def set_shot_random_boundary(self, base_seed, **kw):
        self.seeds.append(base_seed)

    def gradient_shots_dev(self, shots_, ptr):
        off = 0
        for s in shots_:
            n = self.shot_nrec(s) * self.nt
            r = self._view(ptr + 4 * off, n).astype(np.float64)
            pattern = np.cos(0.1 * (s + 1) * np.arange(self.img.size)).reshape(self.img.shape)
            self.img += (pattern * r.sum()).astype(np.float32)
            self.ill += np.float32(s + 1)
            off += n

    def get_accumulators_dev(self, img, ill):
        self._view(img, self.img.size)[:] = self.img.ravel()
        self._view(ill, self.ill.size)[:] = self.ill.ravel()

    def set_accumulators_dev(self, img, ill):
        self.img[:] = self._view(img, self.img.size).reshape(self.img.shape)
        self.ill[:] = self._view(ill, self.ill.size).reshape(self.ill.shape)

    def gradient_post(self, zmask):
        nb = self.nb
        g = self.img[nb:-nb, nb:-nb, nb:-nb] / self.ill[nb:-nb, nb:-nb, nb:-nb]
        m = float(np.abs(g).max())
        return (g / m).astype(np.float32), m

    def get_accumulators(self):
        return self.img.copy(), self.ill.copy()


def _fwi_case():
    from fwi3d_b200 import synth
    w = synth.small_fwi(0, n=8, nt=16)
    w.nb = 2
    w.src = synth.surface_grid([10.0, 30.0, 50.0], [10.0, 40.0], 10.0)  # 6 shots
    return w


def _fwi_steps(world, rank):
    """Misfit of the start model, one gradient, and the misfit of a second
    model, through fwi.Fwi with world/rank."""
    from fwi3d_b200 import fwi
    w = _fwi_case()
    prob = fwi.Fwi(w, fwi.FwiOptions(batch=2), world=world, rank=rank,
                   contexts=(FakeContext(w), FakeContext(w)), device="cpu")
    f0 = prob.misfit(w.start)
    g, raw, ill, f1 = prob.gradient(w.start)
    f2 = prob.misfit((w.start * 1.01).astype(np.float32))
    return prob.mine, f0, f1, f2, g, raw, ill


def _fwi_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, _fwi_steps(None, None)))  # world and rank from torch.distributed
    finally:
        dist.destroy_process_group()


def test_two_rank_fwi_misfit_and_gradient_equal_one_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fwi_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    one = _fwi_steps(1, 0)
    assert sorted(out[0][0] + out[1][0]) == one[0] == list(range(6))
    assert out[0][0] == [0, 2, 4] and out[1][0] == [1, 3, 5]
    for r in (0, 1):
        for k in (1, 2, 3):  # misfits: FP64 sums over every shot of every rank
            assert abs(out[r][k] - one[k]) <= 1e-12 * abs(one[k]), (r, k)
        assert out[r][1] == out[r][2]  # the gradient reuses the misfit of the same model
        for k in (4, 5, 6):  # gradient, raw gradient, illumination: sums over shots
            np.testing.assert_allclose(out[r][k], one[k], rtol=1e-5, atol=1e-6 * np.abs(one[k]).max())
    np.testing.assert_array_equal(out[0][4], out[1][4])  # every rank takes the same step
