"""Parity of the CUDA path (through the C ABI) with the FP64 oracle.

Each test runs the same seeded inputs through libfwi3d.so and through
oracle/liboracle.so and bounds the relative L2 error; the bounds are the FP32
tolerances stated in tests/cases.py.
"""
import numpy as np
import pytest

import oracle as orc
from cases import TOL_GRAD, TOL_IMAGE, TOL_SEIS, context, indices, interior, oracle_wavelet, rel_l2
from fwi3d_b200 import lib, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    return synth.small_case(n=36, nb=8, nt=140, seed=1)


def _oracle_forward(ctx, w, vpp, abc):
    w64, _ = oracle_wavelet(ctx, w)
    src, rec = indices(w, w.nb)
    seis, P, Q = orc.forward(vpp, w.dh, w.dt, w.nt, ctx.tlag, w64, src[0], rec, abc=abc, nb=w.nb,
                             factor=w.abc_factor)
    return seis, P, Q, w64, src, rec


def test_padding_matches_reference_layout(small):
    w = small
    ctx = context(w, lib.BOUNDARY_ABC)
    ctx.set_velocity(w.vp)
    got = ctx.get_padded_velocity()
    want = orc.expand(w.vp, w.nz, w.nx, w.ny, w.nb)
    assert np.array_equal(got, want.astype(np.float32))


def test_forward_abc_matches_oracle(small):
    w = small
    w.abc_factor = 0.02
    ctx = context(w, lib.BOUNDARY_ABC)
    ctx.set_velocity(w.vp)
    seis = ctx.model_shots([0])[0]
    vpp = ctx.get_padded_velocity()
    ref, *_ = _oracle_forward(ctx, w, vpp, abc=True)
    err = rel_l2(seis, ref)
    assert err < TOL_SEIS, f"ABC seismogram rel L2 {err:.3e}"
    assert np.all(seis[:, 0] == 0.0)


def test_forward_rbc_matches_oracle(small):
    w = small
    ctx = context(w, lib.BOUNDARY_RBC)
    ctx.set_velocity(w.vp)
    ctx.apply_random_boundary(kind=0, ratio=30.0, varVp=300.0, seed=7)
    vpp = ctx.get_padded_velocity()
    seis = ctx.model_shots([0])[0]
    ref, *_ = _oracle_forward(ctx, w, vpp, abc=False)
    err = rel_l2(seis, ref)
    assert err < TOL_SEIS, f"RBC seismogram rel L2 {err:.3e}"


@pytest.mark.parametrize("pad", [False, True])
@pytest.mark.parametrize("grad,with_dy", [(False, False), (True, False), (True, True)])
def test_backward_matches_oracle(small, grad, with_dy, pad):
    """pad: the reference's accumulation over every updated cell; otherwise
    the physical box accumulates and the pad keeps its zeros."""
    w = small
    flags = (lib.FLAG_GRAD_DY if with_dy else 0) | (lib.FLAG_PAD_ACCUMULATE if pad else 0)
    ctx = context(w, lib.BOUNDARY_RBC, flags=flags)
    ctx.set_velocity(w.vp)
    ctx.apply_random_boundary(kind=1, ratio=0.3, seed=3)
    vpp = ctx.get_padded_velocity()
    # data: the seismogram of a perturbed model (the reflection residual)
    rng = np.random.default_rng(5)
    data = rng.standard_normal((len(w.rec), w.nt)).astype(np.float32)
    if grad:
        ctx.gradient_shots([0], data)
    else:
        ctx.rtm_shots([0], data)
    img, ill = ctx.get_accumulators()
    _, P, Q, w64, src, rec = _oracle_forward(ctx, w, vpp, abc=False)
    rimg, rill, _, _ = orc.backward(vpp, w.dh, w.dt, w.nt, ctx.tlag, rec, data, P, Q, mode=int(grad),
                                    with_dy=with_dy, w=w64, src=src[0])
    if not pad:
        box = np.zeros(img.shape, bool)
        box[w.nb:-w.nb, w.nb:-w.nb, w.nb:-w.nb] = True
        assert not img[~box].any() and not ill[~box].any()
        img, ill, rimg, rill = (interior(a, w.nb) for a in (img, ill, rimg, rill))
    e_img, e_ill = rel_l2(img, rimg), rel_l2(ill, rill)
    tol = TOL_GRAD if grad else TOL_IMAGE
    assert e_img < tol and e_ill < tol, f"image {e_img:.3e} illum {e_ill:.3e}"


def test_rtm_image_post(small):
    w = small
    ctx = context(w, lib.BOUNDARY_RBC)
    ctx.set_velocity(w.vp)
    data = np.random.default_rng(2).standard_normal((len(w.rec), w.nt)).astype(np.float32)
    ctx.rtm_shots([0], data)
    img, ill = ctx.get_accumulators()
    got = ctx.rtm_image()
    want = orc.rtm_post(img, ill, w.nz, w.nx, w.ny, w.nb, w.dh)
    assert rel_l2(got, want) < 1e-5


def test_gradient_post(small):
    w = small
    ctx = context(w, lib.BOUNDARY_RBC)
    ctx.set_velocity(w.vp)
    data = np.random.default_rng(4).standard_normal((len(w.rec), w.nt)).astype(np.float32)
    ctx.gradient_shots([0], data)
    g, ill = ctx.get_accumulators()
    got, gmax = ctx.gradient_post(zmask=40.0)
    want, rgmax = orc.gradient_post(g, ill, w.nz, w.nx, w.ny, w.nb, w.dh, 40.0)
    assert rel_l2(got, want) < 1e-5
    assert abs(gmax - rgmax) <= 1e-5 * rgmax


def test_batched_shots_equal_single_shots():
    w = synth.small_case(n=30, nb=6, nt=100, seed=2)
    w.src = np.array([[60.0, 70.0, 20.0], [150.0, 120.0, 30.0], [220.0, 200.0, 20.0]], np.float32)
    single = context(w, lib.BOUNDARY_RBC, max_batch=1)
    batch = context(w, lib.BOUNDARY_RBC, max_batch=3)
    for c in (single, batch):
        c.set_velocity(w.vp)
    a = single.model_shots([0, 1, 2])
    b = batch.model_shots([0, 1, 2])
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    data = np.random.default_rng(0).standard_normal((3 * len(w.rec), w.nt)).astype(np.float32)
    single.rtm_shots([0, 1, 2], data)
    batch.rtm_shots([0, 1, 2], data)
    ia, la = single.get_accumulators()
    ib, lb = batch.get_accumulators()
    assert rel_l2(ib, ia) < 1e-6 and rel_l2(lb, la) < 1e-6


def test_every_tile_gives_identical_results():
    w = synth.small_case(n=30, nb=6, nt=80, seed=3)
    ctx = context(w, lib.BOUNDARY_RBC)
    ctx.set_velocity(w.vp)
    data = np.random.default_rng(1).standard_normal((len(w.rec), w.nt)).astype(np.float32)
    base = None
    for t in range(len(lib.tile_table())):
        ctx.set_tiles(t, t)
        seis = ctx.model_shots([0])[0]
        ctx.reset_accumulators()
        ctx.rtm_shots([0], data)
        img, ill = ctx.get_accumulators()
        if base is None:
            base = (seis, img, ill)
        else:
            assert np.array_equal(seis, base[0]), f"tile {t} seismogram differs"
            assert np.array_equal(img, base[1]) and np.array_equal(ill, base[2]), f"tile {t} image differs"


def test_source_subtraction_restores_the_forward_field(small):
    """With the source removed while rebuilding, the back-propagated source
    field at t=0 returns to the initial state (up to FP32 round-off)."""
    w = small
    ctx = context(w, lib.BOUNDARY_RBC, flags=lib.FLAG_SUBTRACT_SOURCE)
    ctx.set_velocity(w.vp)
    vpp = ctx.get_padded_velocity()
    data = np.zeros((len(w.rec), w.nt), np.float32)
    ctx.rtm_shots([0], data)
    _, ill = ctx.get_accumulators()
    _, P, Q, w64, src, rec = _oracle_forward(ctx, w, vpp, abc=False)
    _, rill, _, _ = orc.backward(vpp, w.dh, w.dt, w.nt, ctx.tlag, rec, data, P, Q, mode=0,
                                 subtract_src=True, w=w64, src=src[0])
    assert rel_l2(interior(ill, w.nb), interior(rill, w.nb)) < TOL_IMAGE


def test_residual_fp64():
    w = synth.small_case(n=20, nb=4, nt=50)
    ctx = context(w, lib.BOUNDARY_ABC)
    rng = np.random.default_rng(9)
    obs = rng.standard_normal(200_003).astype(np.float32)
    cal = rng.standard_normal(200_003).astype(np.float32)
    res, s = ctx.residual(obs, cal)
    assert np.array_equal(res, obs - cal)
    want = float(np.sum((obs - cal).astype(np.float64) ** 2))
    assert abs(s - want) <= 1e-12 * want


def test_cfl_violation_is_reported():
    w = synth.small_case(n=20, nb=4, nt=50)
    ctx = context(w, lib.BOUNDARY_ABC)
    with pytest.raises(lib.FwiError) as e:
        ctx.set_velocity(np.full(w.vp.shape, 9000.0, np.float32))
    assert e.value.code == 7


def test_bounded_wait_reports_a_timeout_and_the_context_survives():
    """A wait on an mbarrier that nothing completes gives up after its limit
    and surfaces as FWI_ERR_TIMEOUT; the next call works normally."""
    w = synth.small_case(n=20, nb=4, nt=40)
    ctx = context(w, lib.BOUNDARY_RBC)
    assert ctx.lib.fwi_selftest_bounded_wait(ctx.h, 50) == 4
    ctx.set_velocity(w.vp)
    seis = ctx.model_shots([0])[0]
    assert np.all(np.isfinite(seis)) and np.abs(seis).max() > 0
