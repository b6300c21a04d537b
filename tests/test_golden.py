"""Golden vectors of the reference's own CUDA build (tests/golden/*.npz,
produced by tests/golden/make_golden.py on a B200) pin the FP64 oracle
(CPU tests) and the CUDA library (GPU tests)."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import golden_cases as gc  # noqa: E402
import oracle as orc  # noqa: E402
from cases import rel_l2  # noqa: E402

# Reference build vs oracle: the reference stores FP32 and evaluates its
# stencil in FP64; the oracle is FP64 throughout.
TOL_REF_SEIS = 2e-5
TOL_REF_ACC = 1e-4


@pytest.fixture(scope="module")
def w():
    return gc.workload()


def _oracle_inputs(w):
    wl, tl = orc.wavelet(w.nt, w.dt, w.fmax)
    nzz, nxx = w.nz + 2 * w.nb, w.nx + 2 * w.nb

    def flat(p):
        return orc.flat_index(orc.grid_index(float(p[2]), w.dh, w.nb), orc.grid_index(float(p[0]), w.dh, w.nb),
                              orc.grid_index(float(p[1]), w.dh, w.nb), nzz, nxx)

    return wl, tl, flat(w.src[0]), np.array([flat(r) for r in w.rec], np.int64)


def test_fixtures_present():
    for n in ("ref_abc_forward", "ref_rbc_rtm", "ref_rbc_gradient"):
        assert (gc.HERE / f"{n}.npz").exists(), f"missing golden fixture {n}"


def test_reference_is_deterministic_on_this_grid():
    for n in ("ref_abc_forward", "ref_rbc_rtm", "ref_rbc_gradient"):
        assert float(gc.load(n)["spread"]) < 1e-5


def test_oracle_matches_reference_modeling(w):
    g = gc.load("ref_abc_forward")
    wl, tl, src, rec = _oracle_inputs(w)
    assert tl == int(g["tlag"])
    vpp = orc.expand(w.vp, w.nz, w.nx, w.ny, w.nb)
    seis, _, _ = orc.forward(vpp, w.dh, w.dt, w.nt, tl, wl, src, rec, abc=True, nb=w.nb, factor=gc.ABC_FACTOR)
    assert rel_l2(seis, g["seis"]) < TOL_REF_SEIS


@pytest.mark.parametrize("name,mode", [("ref_rbc_rtm", 0), ("ref_rbc_gradient", 1)])
def test_oracle_matches_reference_backward(w, name, mode):
    g = gc.load(name)
    wl, tl, src, rec = _oracle_inputs(w)
    vpr = gc.random_pad(w)
    seis, P, Q = orc.forward(vpr, w.dh, w.dt, w.nt, tl, wl, src, rec)
    assert rel_l2(seis, g["seis"]) < TOL_REF_SEIS
    img, ill, _, _ = orc.backward(vpr, w.dh, w.dt, w.nt, tl, rec, gc.adjoint_data(w), P, Q, mode=mode)
    for k, s in enumerate(gc.slices(img)):
        assert rel_l2(s, g[f"image{k}"]) < TOL_REF_ACC
    for k, s in enumerate(gc.slices(ill)):
        assert rel_l2(s, g[f"illum{k}"]) < TOL_REF_ACC
    assert abs(np.linalg.norm(img) - float(g["image_norm"])) < TOL_REF_ACC * float(g["image_norm"])


@pytest.mark.gpu
@pytest.mark.parametrize("name,mode", [("ref_rbc_rtm", 0), ("ref_rbc_gradient", 1)])
def test_library_matches_reference_backward(w, name, mode):
    from cases import context
    from fwi3d_b200 import lib
    g = gc.load(name)
    # the reference's padded accumulators: accumulate in the pad too
    ctx = context(w, lib.BOUNDARY_RBC, flags=lib.FLAG_PAD_ACCUMULATE)
    ctx.set_padded_velocity(gc.random_pad(w))
    seis = ctx.model_shots([0])[0]
    assert rel_l2(seis, g["seis"]) < TOL_REF_SEIS
    data = gc.adjoint_data(w)
    (ctx.gradient_shots if mode else ctx.rtm_shots)([0], data)
    img, ill = ctx.get_accumulators()
    for k, s in enumerate(gc.slices(img)):
        assert rel_l2(s, g[f"image{k}"]) < TOL_REF_ACC
    for k, s in enumerate(gc.slices(ill)):
        assert rel_l2(s, g[f"illum{k}"]) < TOL_REF_ACC


@pytest.mark.gpu
def test_library_matches_reference_modeling(w):
    from cases import context
    from fwi3d_b200 import lib
    g = gc.load("ref_abc_forward")
    ctx = context(w, lib.BOUNDARY_ABC, abc_factor=gc.ABC_FACTOR)
    ctx.set_velocity(w.vp)
    seis = ctx.model_shots([0])[0]
    assert rel_l2(seis, g["seis"]) < TOL_REF_SEIS
