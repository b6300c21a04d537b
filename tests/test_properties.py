"""Size-independent properties at the benchmark sizes, where the FP64 oracle
is too slow to run in a test: linearity of migration in the data, batching
that changes nothing, determinism of the random boundary."""
import numpy as np
import pytest

from cases import rel_l2
from fwi3d_b200 import lib, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rtm():
    """The batched-RTM workload (201^3 model, 301^3 padded, nt = 2001): one
    context with the migration model and a fixed random pad."""
    w = synth.rtm_201()
    ctx = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC)
    ctx.set_geometry(w.src, w.rec, w.rec_first, w.rec_count)
    ctx.set_velocity(w.start)
    ctx.apply_random_boundary(seed=11, **w.rbc)
    return w, ctx


def _image(ctx, shot, data):
    ctx.reset_accumulators()
    ctx.rtm_shots([shot], data)
    return ctx.get_accumulators()


def test_rtm_image_is_linear_in_the_data_at_full_size(rtm):
    w, ctx = rtm
    shot = 27
    n = ctx.shot_nrec(shot)
    rng = np.random.default_rng(0)
    d1 = rng.standard_normal((n, w.nt)).astype(np.float32)
    d2 = rng.standard_normal((n, w.nt)).astype(np.float32)
    i1, l1 = _image(ctx, shot, d1)
    i2, l2 = _image(ctx, shot, d2)
    i3, l3 = _image(ctx, shot, (d1 + 2.0 * d2).astype(np.float32))
    assert rel_l2(i3, i1 + 2.0 * i2) < 1e-4
    # the illumination depends on the source field only
    assert np.array_equal(l1, l2) and np.array_equal(l1, l3)


def test_random_boundary_is_deterministic_in_its_seed(rtm):
    w, ctx = rtm
    a = ctx.get_padded_velocity()
    ctx.apply_random_boundary(seed=12, **w.rbc)
    b = ctx.get_padded_velocity()
    ctx.apply_random_boundary(seed=11, **w.rbc)
    c = ctx.get_padded_velocity()
    assert np.array_equal(a, c) and not np.array_equal(a, b)
    k = w.nb + 1
    assert np.array_equal(a[k:-k, k:-k, k:-k], b[k:-k, k:-k, k:-k])
    assert a.max() <= 0.98 * 2 / np.sqrt(3 * 6.5015873) * w.dh / w.dt * (1 + 1e-5)


def test_modeling_batches_change_nothing_at_full_size():
    """The plain-modeling workload (101^3, 201^3 padded, nt = 1001) with a
    second shot: two shots in one launch equal two single-shot launches bit
    for bit."""
    w = synth.modeling_101()
    w.src = np.array([[500.0, 500.0, 10.0], [250.0, 700.0, 30.0]], np.float32)
    out = []
    for B in (1, 2):
        ctx = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC, 0.0, B)
        ctx.set_geometry(w.src, w.rec)
        ctx.set_velocity(w.vp)
        ctx.apply_random_boundary(seed=3, **w.rbc)
        out.append(ctx.model_shots([0, 1]))
        ctx.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
    assert np.all(np.isfinite(out[0][0])) and np.abs(out[0][0]).max() > 0
