"""Batched shots with a random boundary per shot (fwi_set_shot_random_boundary):
every batch slot propagates through its own velocity slot, so shots with
different pads share one launch, and a shot's result does not depend on the
batch it runs in.  The reference builds a new pad per shot and runs shots
one at a time (src/migration/migration.cu:49-80, src/migration_main.cpp:13-19)."""
import numpy as np
import pytest

from cases import rel_l2
from fwi3d_b200 import lib, synth

pytestmark = pytest.mark.gpu

RBC = dict(kind=0, ratio=40.0, varVp=400.0)
BASE = 100


def _case():
    w = synth.small_case(n=30, nb=8, nt=100, seed=2)
    w.src = np.array([[60.0, 70.0, 20.0], [150.0, 120.0, 30.0], [220.0, 200.0, 20.0], [100.0, 250.0, 30.0]],
                     np.float32)
    return w


def _ctx(w, B, flags=0):
    c = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC, 0.0, B, flags)
    c.set_geometry(w.src, w.rec)
    c.set_velocity(w.vp)
    return c


def test_per_shot_pads_equal_one_pad_per_call():
    """B = 1 with per-shot pads is exactly the reference's loop: a new pad,
    then one shot."""
    w = _case()
    data = np.random.default_rng(0).standard_normal((4 * len(w.rec), w.nt)).astype(np.float32)
    loop = _ctx(w, 1)
    seis_loop = []
    for s in range(4):
        loop.apply_random_boundary(seed=BASE + s, **RBC)
        seis_loop.append(loop.model_shots([s])[0])
        loop.rtm_shots([s], data[s * len(w.rec):(s + 1) * len(w.rec)])
    mode = _ctx(w, 1)
    mode.set_shot_random_boundary(base_seed=BASE, **RBC)
    seis_mode = mode.model_shots([0, 1, 2, 3])
    mode.rtm_shots([0, 1, 2, 3], data)
    for a, b in zip(seis_loop, seis_mode):
        assert np.array_equal(a, b)
    for a, b in zip(loop.get_accumulators(), mode.get_accumulators()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("B", [2, 4])
def test_batched_per_shot_pads_equal_single_shots(B):
    w = _case()
    data = np.random.default_rng(1).standard_normal((4 * len(w.rec), w.nt)).astype(np.float32)
    out = {}
    for b in (1, B):
        c = _ctx(w, b, lib.FLAG_GRAD_DY | lib.FLAG_SUBTRACT_SOURCE)
        c.set_shot_random_boundary(base_seed=BASE, **RBC)
        seis = c.model_shots([3, 1, 0, 2])
        c.rtm_shots([0, 1, 2, 3], data)
        img, ill = c.get_accumulators()
        c.reset_accumulators()
        c.gradient_shots([0, 1, 2, 3], data)
        grad, gill = c.get_accumulators()
        out[b] = (seis, img, ill, grad, gill)
        c.close()
    for x, y in zip(out[1][0], out[B][0]):
        assert np.array_equal(x, y)  # modeling: no accumulation, bit for bit
    for x, y in zip(out[1][1:], out[B][1:]):
        assert rel_l2(y, x) < 1e-6  # sums over shots in another order


def test_turning_per_shot_pads_off_restores_the_clean_model():
    w = _case()
    c = _ctx(w, 3)
    clean = c.get_padded_velocity()
    c.set_shot_random_boundary(base_seed=BASE, **RBC)
    c.model_shots([0, 1, 2])
    c.clear_shot_random_boundary()
    assert np.array_equal(c.get_padded_velocity(), clean)
    a = c.model_shots([0, 1])
    ref = _ctx(w, 1)
    for x, y in zip(a, ref.model_shots([0, 1])):
        assert np.array_equal(x, y)
