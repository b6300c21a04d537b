"""The random-boundary pad against its NumPy restatement (oracle/rbc_oracle.py)
and against the reference's recipe (src/modeling/modeling.cu:558-673).

  - the counter-based hash has SplitMix64's published output (CPU);
  - the background pass (edge value + ramped Gaussian noise per pad axis, or
    the ramped uniform relative perturbation) is bit-exact;
  - the blob pass, replayed from the library's own blob list, matches to a
    few FP32 ulps (expf on the device, exp on the host), clamp included;
  - the blob list has the reference's distributions: radius U(0.2 r, r),
    amplitude U(0.5 varVp, varVp), sign negative with probability 1/3,
    centres outside the inner half-pad box, Poisson-disk spacing >= r;
  - the background noise over one pad face is N(0, 1) scaled by
    (1 - depth/nb) varVp.
"""
import numpy as np
import pytest

import oracle as orc
import rbc_oracle as ro
from fwi3d_b200 import lib, synth


def test_splitmix64_known_answers():
    # SplitMix64 with state 0 (Steele, Lea and Flood; the reference
    # implementation's first three outputs): mix(k * golden) for k = 1, 2, 3
    g = 0x9E3779B97F4A7C15
    got = ro.splitmix64(np.array([0, g, (2 * g) % 2**64], np.uint64))
    assert [int(x) for x in got] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_uniforms_are_in_the_open_unit_interval_and_flat():
    u = ro.uniform01(7, 1, np.arange(200_000, dtype=np.uint64))
    assert u.dtype == np.float32 and u.min() > 0 and u.max() < 1
    assert abs(float(u.mean()) - 0.5) < 3e-3
    n = ro.normal01(7, 1, np.arange(200_000, dtype=np.uint64))
    assert abs(float(n.mean())) < 0.01 and abs(float(n.std()) - 1.0) < 0.01


def _ctx(n=40, nb=20):
    w = synth.small_case(n=n, nb=nb, nt=20, seed=6)
    ctx = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC)
    ctx.set_velocity(w.vp)
    clean = ctx.get_padded_velocity()
    return w, ctx, clean


@pytest.mark.gpu
@pytest.mark.parametrize("kind,ratio,varVp", [(0, 0.0, 600.0), (1, 0.35, 0.0)])
def test_background_pass_is_bit_exact(kind, ratio, varVp):
    w, ctx, clean = _ctx()
    assert np.array_equal(clean, orc.expand(w.vp, w.nz, w.nx, w.ny, w.nb).astype(np.float32))
    for seed in (3, 2**40 + 11):
        ctx.apply_random_boundary(kind=kind, ratio=ratio, varVp=varVp, seed=seed)
        got = ctx.get_padded_velocity()
        vlo, vhi, blobs = ctx.random_boundary_recipe(kind=kind, ratio=ratio, varVp=varVp, seed=seed)
        assert len(blobs) == 0
        want = ro.background(clean, w.nb, kind, ratio, varVp, vlo, vhi, seed)
        diff = np.count_nonzero(got != want)
        print(f"kind {kind} seed {seed}: {diff} of {got.size} cells differ")
        assert diff == 0
        nb = w.nb
        assert np.array_equal(got[nb:-nb, nb:-nb, nb:-nb], clean[nb:-nb, nb:-nb, nb:-nb])


@pytest.mark.gpu
def test_blob_pass_and_clamp_match_the_restatement():
    w, ctx, clean = _ctx()
    rbc = dict(kind=0, ratio=40.0, varVp=500.0)
    ctx.apply_random_boundary(seed=21, **rbc)
    got = ctx.get_padded_velocity()
    vlo, vhi, blobs = ctx.random_boundary_recipe(seed=21, **rbc)
    assert len(blobs) > 50
    bg = ro.background(clean, w.nb, 0, rbc["ratio"], rbc["varVp"], vlo, vhi, 21)
    want = ro.blob_pass(bg, w.nb, w.dh, blobs, vlo, vhi)
    d = np.abs(got.astype(np.float64) - want)
    print(f"{len(blobs)} blobs; max |diff| {d.max():.3e} m/s, cells > 2e-3 m/s: {np.count_nonzero(d > 2e-3)}")
    assert d.max() < 1e-2
    assert np.count_nonzero(d > 2e-3) <= 1e-4 * d.size
    # the blobs changed the pad: the restatement without them is far off
    assert np.abs(got.astype(np.float64) - bg).max() > 50.0
    assert got.min() >= vlo and got.max() <= vhi


@pytest.mark.gpu
def test_blob_list_has_the_reference_distributions():
    w = synth.small_case(n=100, nb=50, nt=20, seed=2)
    ctx = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC)
    ctx.set_velocity(w.vp)
    ratio, varVp = 60.0, 800.0
    vlo, vhi, b = ctx.random_boundary_recipe(kind=0, ratio=ratio, varVp=varVp, seed=5)
    n = len(b)
    assert n > 1000
    x, y, z, r, amp = b.T.astype(np.float64)
    # radius U(0.2 r, r), amplitude U(0.5 varVp, varVp) (modeling.cu:585-586)
    assert r.min() >= 0.2 * ratio * (1 - 1e-6) and r.max() <= ratio * (1 + 1e-6)
    assert abs(r.mean() - 0.6 * ratio) < 4 * (0.8 * ratio / np.sqrt(12)) / np.sqrt(n)
    a = np.abs(amp)
    assert a.min() >= 0.5 * varVp * (1 - 1e-6) and a.max() <= varVp * (1 + 1e-6)
    assert abs(a.mean() - 0.75 * varVp) < 4 * (0.5 * varVp / np.sqrt(12)) / np.sqrt(n)
    # sign negative with probability 1/3 (rand() % 3 == 0, modeling.cu:588)
    p = float(np.mean(amp < 0))
    assert abs(p - 1 / 3) < 4 * np.sqrt((1 / 3) * (2 / 3) / n), p
    # centres outside the inner box shrunk by half the pad (modeling.cu:571-577)
    h = 0.5 * w.nb * w.dh
    xm, ym, zm = (ctx.nxx - 1) * w.dh, (ctx.nyy - 1) * w.dh, (ctx.nzz - 1) * w.dh
    inner = (x > h) & (x < xm - h) & (y > h) & (y < ym - h) & (z > h) & (z < zm - h)
    assert not inner.any()
    assert x.min() >= 0 and x.max() <= xm and y.min() >= 0 and y.max() <= ym and z.min() >= 0 and z.max() <= zm
    # Poisson-disk spacing: no two centres closer than r (admin.cpp:105-207)
    from scipy.spatial import cKDTree
    d, _ = cKDTree(np.stack([x, y, z], 1)).query(np.stack([x, y, z], 1), k=2)
    assert d[:, 1].min() >= ratio * (1 - 1e-5)
    # and the sampling fills the shell: every pad cell of an outer face is
    # within 2 r of a centre
    gx = np.arange(0, xm, 4 * w.dh)
    face = np.stack(np.meshgrid(gx, gx, [0.0], indexing="ij"), -1).reshape(-1, 3)
    dist, _ = cKDTree(np.stack([x, y, z], 1)).query(face)
    assert dist.max() <= 2 * ratio * (1 + 1e-5)


@pytest.mark.gpu
def test_background_noise_is_ramped_gaussian():
    w, ctx, clean = _ctx(n=60, nb=30)
    varVp = 10.0  # small: the clamp never acts
    ctx.apply_random_boundary(kind=0, ratio=0.0, varVp=varVp, seed=9)
    got = ctx.get_padded_velocity().astype(np.float64)
    nb = w.nb
    # x-face cells only (z and y inside): noise = (1 - j/nb) varVp N(0, 1)
    sl = got[nb:-nb, :nb, nb:-nb] - clean[nb:-nb, :nb, nb:-nb]
    ramp = 1.0 - np.arange(nb) / nb
    z = sl / (ramp[None, :, None] * varVp)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01, (z.mean(), z.std())
