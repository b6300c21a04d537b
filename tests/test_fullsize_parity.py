"""Parity at the benchmark configurations' full grid sizes.

Each test runs one configuration's grid through libfwi3d.so and through the
checkers on identical inputs (the same padded velocity, sources, receivers and
data), and prints its relative L2 errors beside the bounds of tests/cases.py:

  plain modeling      101^3 model + 50-cell pad (201^3 padded), nt = 1001,
                      51 x 51 receivers, source at the centre 10 m deep:
                      seismogram vs the FP64 oracle and vs the reference's own
                      CUDA build, random boundary and Cerjan boundary;
  batched RTM shot    201^3 model + 50-cell pad (301^3 padded), one interior
                      shot with its 121 x 121 receiver patch: image and
                      illumination vs the reference build at the full
                      nt = 2001 (N = 2120 steps), and vs the FP64 oracle at
                      nt = 1001 (the oracle needs about a minute for that);
  mixed-precision     401 x 401 x 201 at 12.5 m + 41-cell pad (483 x 483 x 283
  gradient            padded), one shot, time axis shortened to nt = 200 so
                      that the oracle finishes: seismograms (true and start
                      model), misfit, raw gradient and illumination, the
                      post-processed gradient and the parabolic step vs the
                      FP64 oracle; the raw gradient also vs the reference build.

Images, gradients and illumination are compared over the physical box: the
library accumulates them there only, the part that the post-processing reads.

The Cerjan case compares the reference build with ours only up to the
reference's own race (it damps P in place while neighbouring blocks read it).

The reference-build legs are skipped where oracle/_ref was not built.
"""
import numpy as np
import pytest

import oracle as orc
from cases import TOL_GRAD, TOL_IMAGE, TOL_SEIS, indices, interior, oracle_wavelet, rel_l2
from fwi3d_b200 import lib, synth

pytestmark = pytest.mark.gpu

# Misfit: a sum of squares of differences of nearly equal seismograms, so its
# relative error is larger than the seismograms'.  Parabolic step of the line
# search: the vertex is a ratio of first and second differences of three such
# misfits that differ by a few per cent, which amplifies their error again.
TOL_MISFIT = 2e-3
TOL_STEP = 2e-2

needs_ref = pytest.mark.skipif(not orc.ref_available(), reason="oracle/_ref not built")


def _report(name, err, bound):
    print(f"{name}: rel L2 {err:.3e} (bound {bound:.0e})")
    assert err < bound, f"{name}: {err:.3e} >= {bound:.0e}"


def _ctx(w, boundary, flags=0):
    ctx = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, boundary, w.abc_factor, 1, flags)
    ctx.set_geometry(w.src, w.rec, w.rec_first, w.rec_count)
    return ctx


def _one_shot(w, s):
    """Workload restricted to shot s (its own receiver range)."""
    if w.rec_first is not None:
        f, c = int(w.rec_first[s]), int(w.rec_count[s])
        w.rec = w.rec[f:f + c]
        w.rec_first = w.rec_count = None
    w.src = w.src[s:s + 1]
    return w


# ---------------------------------------------------------------------------
# plain modeling, full size
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def modeling_case(tmp_path_factory):
    w = synth.modeling_101()
    params = orc.write_reference_setup(tmp_path_factory.mktemp("c0"), w.nz, w.nx, w.ny, w.dh, w.nt, w.dt,
                                       w.fmax, w.nb, w.src, w.rec, abc_factor=w.abc_factor)
    return w, params


@pytest.mark.parametrize("abc", [False, True], ids=["random-boundary", "cerjan"])
def test_plain_modeling_full_size(modeling_case, abc):
    w, params = modeling_case
    ctx = _ctx(w, lib.BOUNDARY_ABC if abc else lib.BOUNDARY_RBC)
    ctx.set_velocity(w.vp)
    if not abc:
        ctx.apply_random_boundary(seed=1, **w.rbc)
    vpp = ctx.get_padded_velocity()
    ours = ctx.model_shots([0])[0]
    w64, _ = oracle_wavelet(ctx, w)
    src, rec = indices(w, w.nb)
    ref64, _, _ = orc.forward(vpp, w.dh, w.dt, w.nt, ctx.tlag, w64, src[0], rec, abc=abc, nb=w.nb,
                              factor=w.abc_factor)
    tag = "cerjan" if abc else "random boundary"
    _report(f"plain modeling 201^3, {tag}: seismogram vs FP64 oracle", rel_l2(ours, ref64), TOL_SEIS)
    assert np.all(ours[:, 0] == 0.0) and np.abs(ours).max() > 0
    if orc.ref_available():
        r = orc.ref_run(params, vpp, abc=abc)
        assert r["tlag"] == ctx.tlag
        if not abc:
            _report(f"plain modeling 201^3, {tag}: seismogram vs reference build", rel_l2(ours, r["seis"]),
                    TOL_SEIS)
            _report(f"plain modeling 201^3, {tag}: reference build vs FP64 oracle", rel_l2(r["seis"], ref64),
                    TOL_SEIS)
        else:
            # The reference damps P in place while neighbouring blocks still read
            # it for their stencils (src/modeling/modeling.cu:374-380); with the
            # 16k blocks of this grid that race is live, so the reference build
            # is not reproducible here and is not the FP64 answer.  Ours is
            # checked against FP64 above; the reference is no closer to ours than
            # it is to FP64.
            r2 = orc.ref_run(params, vpp, abc=abc)
            e_run = rel_l2(r2["seis"], r["seis"])
            e_ref = rel_l2(r["seis"], ref64)
            e_ours = rel_l2(ours, r["seis"])
            print(f"plain modeling 201^3, cerjan: reference build run to run {e_run:.3e}, reference build vs "
                  f"FP64 oracle {e_ref:.3e}, ours vs reference build {e_ours:.3e}")
            assert e_ours <= e_ref * 1.01 + TOL_SEIS
    ctx.close()


# ---------------------------------------------------------------------------
# one batched-RTM shot, full size
# ---------------------------------------------------------------------------
RTM_SHOT = 27  # an interior shot: its receiver patch is not clipped


def _rtm_shot(nt):
    w = _one_shot(synth.rtm_201(nt=nt), RTM_SHOT)
    ctx = _ctx(w, lib.BOUNDARY_RBC)
    ctx.set_velocity(w.start)
    ctx.apply_random_boundary(seed=11, **w.rbc)
    vpp = ctx.get_padded_velocity()
    data = np.random.default_rng(7).standard_normal((len(w.rec), w.nt)).astype(np.float32)
    ctx.rtm_shots([0], data)
    img, ill = ctx.get_accumulators()
    ctx.close()
    return w, vpp, data, img, ill


@needs_ref
def test_rtm_shot_full_size_vs_reference_build(tmp_path):
    w, vpp, data, img, ill = _rtm_shot(2001)
    assert len(w.rec) == 121 * 121
    params = orc.write_reference_setup(tmp_path, w.nz, w.nx, w.ny, w.dh, w.nt, w.dt, w.fmax, w.nb, w.src, w.rec)
    r = orc.ref_run(params, vpp, abc=False, backward=1, adj=data, want_acc=True)
    assert r["tlag"] + w.nt == 2120
    nb = w.nb
    _report("RTM shot 301^3, N = 2120: image vs reference build",
            rel_l2(interior(img, nb), interior(r["image"], nb)), TOL_IMAGE)
    _report("RTM shot 301^3, N = 2120: illumination vs reference build",
            rel_l2(interior(ill, nb), interior(r["illum"], nb)), TOL_IMAGE)


def test_rtm_shot_full_grid_vs_oracle():
    nt = 1001
    w, vpp, data, img, ill = _rtm_shot(nt)
    ctx = _ctx(w, lib.BOUNDARY_RBC)
    w64, _ = oracle_wavelet(ctx, w)
    src, rec = indices(w, w.nb)
    _, P, Q = orc.forward(vpp, w.dh, w.dt, w.nt, ctx.tlag, w64, src[0], rec)
    oimg, oill, _, _ = orc.backward(vpp, w.dh, w.dt, w.nt, ctx.tlag, rec, data, P, Q, mode=0)
    ctx.close()
    nb = w.nb
    _report(f"RTM shot 301^3, nt = {nt}: image vs FP64 oracle",
            rel_l2(interior(img, nb), interior(oimg, nb)), TOL_IMAGE)
    _report(f"RTM shot 301^3, nt = {nt}: illumination vs FP64 oracle",
            rel_l2(interior(ill, nb), interior(oill, nb)), TOL_IMAGE)


# ---------------------------------------------------------------------------
# mixed-precision gradient grid, shortened time axis
# ---------------------------------------------------------------------------
GRAD_NT = 200
GRAD_SHOT = 5


@pytest.fixture(scope="module")
def gradient_case():
    """Seismograms of the true and the start model, the gradient of the start
    model's residual through one random boundary, on both sides."""
    w = _one_shot(synth.gradient_401(nt=GRAD_NT), GRAD_SHOT)
    abc = _ctx(w, lib.BOUNDARY_ABC)
    w64, _ = oracle_wavelet(abc, w)
    src, rec = indices(w, w.nb)
    out = {"w": w, "abc": abc, "w64": w64, "src": src, "rec": rec}
    for name, v in (("obs", w.vp), ("cal", w.start)):
        abc.set_velocity(v)
        g = abc.model_shots([0])[0]
        o, _, _ = orc.forward(abc.get_padded_velocity(), w.dh, w.dt, w.nt, abc.tlag, w64, src[0], rec,
                              abc=True, nb=w.nb, factor=w.abc_factor)
        out[name] = (g, o)
    res = (out["obs"][0] - out["cal"][0]).astype(np.float32)
    rbc = _ctx(w, lib.BOUNDARY_RBC)
    rbc.set_velocity(w.start)
    rbc.apply_random_boundary(seed=3, **w.rbc)
    vpr = rbc.get_padded_velocity()
    rbc.gradient_shots([0], res)
    out["graw"], out["gill"] = rbc.get_accumulators()
    out["gpost"], out["gmax"] = rbc.gradient_post(w.zmask)
    _, P, Q = orc.forward(vpr, w.dh, w.dt, w.nt, rbc.tlag, w64, src[0], rec)
    out["oimg"], out["oill"], _, _ = orc.backward(vpr, w.dh, w.dt, w.nt, rbc.tlag, rec, res, P, Q, mode=1)
    del P, Q
    out["opost"], out["omax"] = orc.gradient_post(out["oimg"], out["oill"], w.nz, w.nx, w.ny, w.nb, w.dh, w.zmask)
    out["res"], out["vpr"] = res, vpr
    rbc.close()
    return out


def test_gradient_grid_seismograms_and_misfit(gradient_case):
    c = gradient_case
    for name in ("obs", "cal"):
        _report(f"483x483x283, nt = {GRAD_NT}: {name} seismogram vs FP64 oracle", rel_l2(*c[name]), TOL_SEIS)
    f_gpu = c["abc"].residual(c["obs"][0], c["cal"][0])[1]
    f_orc = float(np.sum((c["obs"][1] - c["cal"][1]) ** 2))
    err = abs(f_gpu / f_orc - 1.0)
    print(f"483x483x283: misfit {f_gpu:.6e} vs FP64 oracle {f_orc:.6e}, rel err {err:.3e} (bound {TOL_MISFIT:.0e})")
    assert err < TOL_MISFIT


def test_gradient_grid_raw_gradient(gradient_case):
    c = gradient_case
    nb = c["w"].nb
    _report(f"483x483x283, nt = {GRAD_NT}: raw gradient vs FP64 oracle",
            rel_l2(interior(c["graw"], nb), interior(c["oimg"], nb)), TOL_GRAD)
    _report(f"483x483x283, nt = {GRAD_NT}: illumination vs FP64 oracle",
            rel_l2(interior(c["gill"], nb), interior(c["oill"], nb)), TOL_GRAD)


@needs_ref
def test_gradient_grid_raw_gradient_vs_reference_build(gradient_case, tmp_path):
    c = gradient_case
    w = c["w"]
    params = orc.write_reference_setup(tmp_path, w.nz, w.nx, w.ny, w.dh, w.nt, w.dt, w.fmax, w.nb, w.src, w.rec)
    r = orc.ref_run(params, c["vpr"], abc=False, backward=2, adj=c["res"], want_acc=True)
    nb = w.nb
    _report(f"483x483x283, nt = {GRAD_NT}: raw gradient vs reference build",
            rel_l2(interior(c["graw"], nb), interior(r["image"], nb)), TOL_GRAD)
    _report(f"483x483x283, nt = {GRAD_NT}: illumination vs reference build",
            rel_l2(interior(c["gill"], nb), interior(r["illum"], nb)), TOL_GRAD)


def _illuminated(c):
    """Post-processed gradients of both sides over the cells the source field
    reached (illumination >= 1e-3 of its peak on the oracle side), each
    renormalised there.  With the shortened time axis the rest is noise over
    noise, flushed to zero in FP32 but not in FP64."""
    w = c["w"]
    ill = orc.reduce(c["oill"], w.nz, w.nx, w.ny, w.nb)
    lit = ill >= 1e-3 * ill.max()
    gu = np.where(lit, c["gpost"].astype(np.float64) * c["gmax"], 0.0)
    ou = np.where(lit, c["opost"] * c["omax"], 0.0)
    return gu / np.abs(gu).max(), ou / np.abs(ou).max(), float(lit.mean())


def test_gradient_grid_post_processed_gradient_and_step(gradient_case):
    c = gradient_case
    w = c["w"]
    gpost, opost, frac = _illuminated(c)
    print(f"483x483x283: illuminated fraction {frac:.3f}")
    _report(f"483x483x283, nt = {GRAD_NT}: post-processed gradient vs FP64 oracle", rel_l2(gpost, opost), TOL_GRAD)
    # the reference's parabola through the misfits at 0, 0.02 dm, 0.05 dm
    # (src/inversion/inversion.cu:291-347), each side with its own gradient
    dm = 1.0 / float(w.start.min()) ** 2 - 1.0 / float(w.start.max()) ** 2
    trials = [0.0, 0.02 * dm, 0.05 * dm]
    m = 1.0 / w.start.astype(np.float64) ** 2
    obs_g, obs_o = c["obs"]
    abc = c["abc"]
    # the step 0 trial is the start model itself: its misfits are known
    fg = [abc.residual(obs_g, c["cal"][0])[1]]
    fo = [float(np.sum((obs_o - c["cal"][1]) ** 2))]
    for alpha in trials[1:]:
        vg = (1.0 / np.sqrt(m - alpha * gpost)).astype(np.float32)
        vo = 1.0 / np.sqrt(m - alpha * opost)
        abc.set_velocity(vg)
        fg.append(abc.residual(obs_g, abc.model_shots([0])[0])[1])
        oc, _, _ = orc.forward(orc.expand(vo, w.nz, w.nx, w.ny, w.nb), w.dh, w.dt, w.nt, abc.tlag, c["w64"],
                               c["src"][0], c["rec"], abc=True, nb=w.nb, factor=w.abc_factor)
        fo.append(float(np.sum((obs_o - oc) ** 2)))
    print(f"483x483x283: misfits at 0, 0.02 dm, 0.05 dm: GPU {fg}, FP64 oracle {fo}")
    sg = orc.parabola_step(*trials, *np.sqrt(fg))
    so = orc.parabola_step(*trials, *np.sqrt(fo))
    err = abs(sg / so - 1.0)
    print(f"483x483x283: step {sg:.6e} vs FP64 oracle {so:.6e}, rel err {err:.3e} (bound {TOL_STEP:.0e})")
    assert err < TOL_STEP
