"""Known-answer tests that need no reference output: the stencil's order of
accuracy, the analytic 3-D Green's function of the constant-velocity wave
equation, and a finite-difference check of the misfit gradient.

The FP64 oracle is checked on the CPU; the same checks run through the C ABI
on the GPU at larger sizes.

Source timing (src/modeling/modeling.cu:324-382): at step t the sample w[t]
scaled by 1/dh^3 is added to the current field before the update, and the
seismogram records the current field.  With Q^t the field after injection,
    Q^{t+1} - 2 Q^t + Q^{t-1} = dt^2 v^2 lap(Q^t) + w[t+1]/dh^3 delta_cell,
the centred discretisation of p_tt = v^2 lap p + w(t + dt)/dt^2 delta(x), whose
free-space solution is p(r, t) = w(t + dt - r/v) / (4 pi v^2 dt^2 r).  The
sample n of a trace is p((n + tlag) dt).

Gradient scale: the gradient accumulates dt Pr v^2 (d2x + d2y + d2z) Ps
(src/inversion/inversion.cu:400-468 with the d2y term), with Pr driven by
(obs - cal)/dh^3.  The adjoint-state derivative of J = sum (obs - cal)^2 with
respect to m = 1/v^2 is then 2 dh^3 dt v_rec^2 g, v_rec the velocity at the
receivers.  The reference pairs the adjoint field with the source field of the
same step rather than the next one, a phase error of about omega dt, so the
finite-difference ratio is bounded to [0.85, 1.1] rather than to 1.
"""
import numpy as np
import pytest

import oracle as orc
from fwi3d_b200 import synth


def ricker(tau, fmax):
    """The reference's wavelet (src/modeling/modeling.cu:36-59) at continuous
    time tau, amplitude 1e5, peak fmax/3, delay 2 sqrt(pi)/fmax."""
    t0 = 2.0 * np.sqrt(np.pi) / fmax
    fc = fmax / (3.0 * np.sqrt(np.pi))
    a = np.pi ** 3 * fc ** 2 * (tau - t0) ** 2
    return 1e5 * (1.0 - 2.0 * a) * np.exp(-a)


def greens_trace(r, v, dt, nt, tlag, fmax):
    n = np.arange(nt)
    p = ricker((n + tlag + 1) * dt - r / v, fmax) / (4.0 * np.pi * v * v * dt * dt * r)
    p[0] = 0.0
    return p


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


# --------------------------------------------------------------------------
# stencil: eighth-order accurate, same symbol on every axis
# --------------------------------------------------------------------------
def _symbol(theta, axis, dh=10.0, n=24):
    f = np.zeros((n, n, n))
    shape = [1, 1, 1]
    shape[axis] = n
    f[:] = np.cos(theta * np.arange(n) + 0.3).reshape(shape)
    lap = orc.laplacian(f, dh)[6:18, 6:18, 6:18]
    fs = f[6:18, 6:18, 6:18]
    m = np.abs(fs) > 0.3
    return float(np.mean(lap[m] / fs[m])) * dh * dh


def test_stencil_is_eighth_order_accurate():
    for axis in range(3):
        e = {th: abs(_symbol(th, axis) + th * th) for th in (0.8, 0.4, 0.2)}
        # an 8th-order second derivative has a symbol error ~ theta^10
        assert 900 < e[0.4] / e[0.2] < 1100, e
        assert 700 < e[0.8] / e[0.4] < 1100, e
        assert e[0.8] < 5e-5 * 0.64
    assert _symbol(0.5, 0) == pytest.approx(_symbol(0.5, 1), rel=1e-12)
    assert _symbol(0.5, 0) == pytest.approx(_symbol(0.5, 2), rel=1e-12)


# --------------------------------------------------------------------------
# analytic Green's function
# --------------------------------------------------------------------------
def test_oracle_matches_the_analytic_greens_function():
    n, dh, dt, fmax, v, nt = 81, 5.0, 5e-4, 60.0, 2000.0, 240
    w, tlag = orc.wavelet(nt, dt, fmax)
    c = n // 2
    vpp = np.full((n, n, n), v)
    offs = [(15, 0, 0), (0, 15, 0), (0, 0, 15), (9, 9, 9), (10, 0, 0), (12, 9, 0)]  # (z, x, y) cells
    rec = [orc.flat_index(c + a, c + b, c + d, n, n) for a, b, d in offs]
    seis, _, _ = orc.forward(vpp, dh, dt, nt, tlag, w, orc.flat_index(c, c, c, n, n), rec)
    half = (c - 4) * dh  # distance to the frozen edge cells
    t0 = 2.0 * np.sqrt(np.pi) / fmax
    for k, o in enumerate(offs):
        r = dh * np.sqrt(sum(x * x for x in o))
        ana = greens_trace(r, v, dt, nt, tlag, fmax)
        # compare up to the first edge reflection's arrival (the wavelet is
        # negligible beyond 45 ms from its peak)
        t_refl = (2 * half - max(abs(x) for x in o) * dh) / v + t0 - 0.045
        m = (np.arange(nt) + tlag) * dt < t_refl
        assert m.sum() > 150
        assert rel_l2(seis[k][m], ana[m]) < 3e-3, o
        assert abs(np.abs(seis[k][m]).max() / np.abs(ana[m]).max() - 1) < 1e-3, o


@pytest.mark.gpu
def test_library_matches_the_analytic_greens_function():
    from fwi3d_b200 import lib
    n, nb, dh, dt, fmax, v, nt = 161, 20, 5.0, 5e-4, 60.0, 2000.0, 400
    c = n // 2
    offs = [(15, 0, 0), (0, 25, 0), (0, 0, 40), (20, 20, 20), (-30, 10, 0)]  # (z, x, y) cells
    src = np.array([[c * dh, c * dh, c * dh]], np.float32)
    rec = np.array([[(c + b) * dh, (c + d) * dh, (c + a) * dh] for a, b, d in offs], np.float32)
    # no random pad and no damping: the padded grid is the constant medium
    ctx = lib.Context(n, n, n, nb, dh, nt, dt, fmax, lib.BOUNDARY_RBC, 0.0, 1, 0)
    ctx.set_geometry(src, rec)
    ctx.set_velocity(np.full((n, n, n), v, np.float32))
    seis = ctx.model_shots([0])[0]
    for k, o in enumerate(offs):
        r = dh * np.sqrt(sum(x * x for x in o))
        ana = greens_trace(r, v, dt, nt, ctx.tlag, fmax)
        # the FP64 oracle's error on this grid grows with distance to 0.46 %
        # at 200 m (numerical dispersion); the edge reflections arrive later
        assert rel_l2(seis[k], ana) < 1e-2, o
        assert abs(np.abs(seis[k]).max() / np.abs(ana).max() - 1) < 2e-3, o


# --------------------------------------------------------------------------
# finite-difference check of the gradient
# --------------------------------------------------------------------------
def _gradient_problem(n=64):
    dh = 10.0
    zz = np.arange(n) * dh
    v0 = np.where(zz < 300, 1800.0, 2400.0)[None, None, :] * np.ones((n, n, 1))
    Y, X, Z = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    vt = v0 * (1 + 0.05 * np.exp(-((X - 32) ** 2 + (Y - 30) ** 2 + (Z - 40) ** 2) / (2 * 5.0 ** 2)))
    rng = np.random.default_rng(0)
    blobs = []
    for _ in range(4):
        cz, cx, cy = rng.uniform(20, 44, 3)
        blobs.append(20.0 * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2) / (2 * 4.0 ** 2)))
    return dh, v0, vt, blobs


def _edge_padded(v, nb):
    """The library's padding of the interior of v (edge replication)."""
    return np.pad(v[nb:-nb, nb:-nb, nb:-nb], nb, mode="edge")


def test_oracle_gradient_matches_finite_differences():
    n, nb, dt, fmax, nt = 64, 8, 1e-3, 30.0, 500
    dh, v0, vt, blobs = _gradient_problem(n)
    w, tlag = orc.wavelet(nt, dt, fmax)
    # source and receivers 4 cells below the top of the interior
    src = orc.flat_index(12, 32, 32, n, n)
    rec = np.array([orc.flat_index(12, j, k, n, n) for j in range(8, 56, 4) for k in range(8, 56, 4)])
    crop = (slice(nb, -nb),) * 3

    def seis(v):
        return orc.forward(_edge_padded(v, nb), dh, dt, nt, tlag, w, src, rec)

    obs = seis(vt)[0]
    cal, P, Q = seis(v0)
    g, *_ = orc.backward(v0, dh, dt, nt, tlag, rec, obs - cal, P, Q, mode=1, with_dy=True,
                         subtract_src=True, w=w, src=src)
    scale = 2 * dh ** 3 * dt * 1800.0 ** 2
    for dv in blobs:
        fd = (np.sum((obs - seis(v0 + dv)[0]) ** 2) - np.sum((obs - seis(v0 - dv)[0]) ** 2)) / 2
        pred = scale * np.sum(g[crop] * (-2 * dv[crop] / v0[crop] ** 3))
        assert 0.85 < fd / pred < 1.1, (fd, pred)


@pytest.mark.gpu
def test_library_gradient_matches_finite_differences():
    from fwi3d_b200 import lib
    n, nb, dt, fmax, nt = 48, 8, 1e-3, 30.0, 500
    dh, v0p, vtp, blobs = _gradient_problem(n + 2 * nb)
    crop = (slice(nb, -nb),) * 3
    v0, vt = v0p[crop].astype(np.float32), vtp[crop].astype(np.float32)
    src = np.array([[(32 - nb) * dh, (32 - nb) * dh, 4 * dh]], np.float32)
    g1 = np.arange(8, 56, 4) - nb
    rec = np.array([[j * dh, k * dh, 4 * dh] for j in g1 for k in g1], np.float32)
    # no random pad: the same edge-replicated grid as the oracle's check
    ctx = lib.Context(n, n, n, nb, dh, nt, dt, fmax, lib.BOUNDARY_RBC, 0.0, 1,
                      lib.FLAG_GRAD_DY | lib.FLAG_SUBTRACT_SOURCE)
    ctx.set_geometry(src, rec)

    def seis(v):
        ctx.set_velocity(np.ascontiguousarray(v, np.float32))
        return ctx.model_shots([0])[0].astype(np.float64)

    obs = seis(vt)
    cal = seis(v0)
    ctx.set_velocity(v0)
    ctx.reset_accumulators()
    ctx.gradient_shots([0], [obs - cal])
    g, _ = ctx.get_accumulators()
    g = g[crop].astype(np.float64)
    scale = 2 * dh ** 3 * dt * 1800.0 ** 2
    for dv in blobs:
        dvi = dv[crop]
        fd = (np.sum((obs - seis(v0 + dvi)) ** 2) - np.sum((obs - seis(v0 - dvi)) ** 2)) / 2
        pred = scale * np.sum(g * (-2 * dvi / v0.astype(np.float64) ** 3))
        assert 0.85 < fd / pred < 1.1, (fd, pred)


def _adjoint_case():
    w = synth.small_case(n=16, nb=6, nt=80, seed=12)
    nb = w.nb
    vpp = orc.expand(w.vp, w.nz, w.nx, w.ny, nb)
    wl, tlag = orc.wavelet(w.nt, w.dt, w.fmax)
    nzz, nxx = w.nz + 2 * nb, w.nx + 2 * nb
    flat = lambda p: orc.flat_index(orc.grid_index(float(p[2]), w.dh, nb), orc.grid_index(float(p[0]), w.dh, nb),
                                    orc.grid_index(float(p[1]), w.dh, nb), nzz, nxx)
    src = flat(w.src[0])
    rec = np.array([flat(r) for r in w.rec], np.int64)
    rng = np.random.default_rng(4)
    d = rng.standard_normal((len(rec), w.nt))
    m = np.zeros_like(vpp)
    m[4:-4, 4:-4, 4:-4] = rng.standard_normal(m[4:-4, 4:-4, 4:-4].shape)
    return w, vpp, wl, tlag, src, rec, d, m


def test_imaging_operator_dot_product_identity():
    """<image(d), m> = <d, adjoint(m)> for the RTM imaging operator with the
    source removed while rebuilding (src/migration/migration.cu:61-81,
    119-202): the image is linear in the data, and orc_image_adjoint (Born
    modelling of m scattering the rebuilt source field) is its exact adjoint."""
    w, vpp, wl, tlag, src, rec, d, m = _adjoint_case()
    _, P, Q = orc.forward(vpp, w.dh, w.dt, w.nt, tlag, wl, src, rec)
    img, _, _, _ = orc.backward(vpp, w.dh, w.dt, w.nt, tlag, rec, d, P, Q, mode=0, subtract_src=True, w=wl,
                                src=src)
    adj = orc.image_adjoint(vpp, w.dh, w.dt, w.nt, tlag, rec, P, Q, m, subtract_src=True, w=wl, src=src)
    lhs, rhs = float(np.sum(img * m)), float(np.sum(d * adj))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), abs(rhs)), (lhs, rhs)
    # not a trivial identity: a different model gives a different product
    assert abs(float(np.sum(img * np.roll(m, 1))) - lhs) > 1e-6 * abs(lhs)


@pytest.mark.gpu
def test_library_imaging_operator_is_the_adjoint_of_born_modelling():
    """The library's RTM image (FP32, source removed while rebuilding) against
    the FP64 adjoint of the same operator: <image_gpu(d), m> equals
    <d, adjoint(m)> to FP32 accuracy."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from cases import context, oracle_wavelet
    from fwi3d_b200 import lib
    w, _, _, _, src, rec, d, m = _adjoint_case()
    # the library images the physical box (the pad is cropped away by every
    # post-processing step), so the model perturbation lives there
    nb = w.nb
    box = np.zeros(m.shape, bool)
    box[nb:-nb, nb:-nb, nb:-nb] = True
    m = np.where(box, m, 0.0)
    ctx = context(w, lib.BOUNDARY_RBC, flags=lib.FLAG_SUBTRACT_SOURCE)
    ctx.set_velocity(w.vp)
    ctx.apply_random_boundary(kind=1, ratio=0.3, seed=8)
    vpp = ctx.get_padded_velocity()
    ctx.rtm_shots([0], d.astype(np.float32))
    img, _ = ctx.get_accumulators()
    w64, _ = oracle_wavelet(ctx, w)
    _, P, Q = orc.forward(vpp, w.dh, w.dt, w.nt, ctx.tlag, w64, src, rec)
    adj = orc.image_adjoint(vpp, w.dh, w.dt, w.nt, ctx.tlag, rec, P, Q, m, subtract_src=True, w=w64, src=src)
    lhs = float(np.sum(img.astype(np.float64) * m))
    rhs = float(np.sum(d.astype(np.float32).astype(np.float64) * adj))
    print(f"<image(d), m> = {lhs:.9e}, <d, adjoint(m)> = {rhs:.9e}, rel diff {abs(lhs - rhs) / abs(rhs):.2e}")
    assert abs(lhs - rhs) <= 1e-4 * abs(rhs)
