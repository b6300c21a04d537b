"""The reference's own CUDA kernels (built from its sources into oracle/_ref)
against the FP64 oracle and against libfwi3d.so, on identical injected inputs,
live on the GPU.  Skipped where oracle/_ref was not built (no reference
sources).  The grid is the golden one: large enough that the reference's
racy source injection (src/modeling/modeling.cu:347-348) lands before the
block owning the source runs, so the reference is deterministic."""
import sys
from pathlib import Path
import numpy as np
import pytest

import oracle as orc
from cases import TOL_IMAGE, TOL_SEIS, context, indices, oracle_wavelet, rel_l2
from fwi3d_b200 import lib, synth

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import golden_cases as gc  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not orc.ref_available(), reason="oracle/_ref not built")]


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    w = gc.workload()
    params = orc.write_reference_setup(tmp_path_factory.mktemp("ref"), w.nz, w.nx, w.ny, w.dh, w.nt, w.dt,
                                       w.fmax, w.nb, w.src, w.rec, abc_factor=w.abc_factor)
    return w, params


def test_reference_modeling_abc(case):
    w, params = case
    vpp = orc.expand(w.vp, w.nz, w.nx, w.ny, w.nb).astype(np.float32)
    ref = orc.ref_run(params, vpp, abc=True)
    ctx = context(w, lib.BOUNDARY_ABC)
    ctx.set_velocity(w.vp)
    ours = ctx.model_shots([0])[0]
    w64, _ = oracle_wavelet(ctx, w)
    src, rec = indices(w, w.nb)
    o, _, _ = orc.forward(vpp, w.dh, w.dt, w.nt, ctx.tlag, w64, src[0], rec, abc=True, nb=w.nb,
                          factor=w.abc_factor)
    assert ref["tlag"] == ctx.tlag
    e_ref_orc = rel_l2(ref["seis"], o)
    e_ours_ref = rel_l2(ours, ref["seis"])
    assert e_ref_orc < TOL_SEIS, f"reference vs oracle {e_ref_orc:.3e}"
    assert e_ours_ref < TOL_SEIS, f"ours vs reference {e_ours_ref:.3e}"


@pytest.mark.parametrize("backward", [1, 2])
def test_reference_backward(case, backward):
    w, params = case
    # the reference's padded accumulators: accumulate in the pad too
    ctx = context(w, lib.BOUNDARY_RBC, flags=lib.FLAG_PAD_ACCUMULATE)
    ctx.set_velocity(w.vp)
    ctx.apply_random_boundary(kind=0, ratio=60.0, varVp=300.0, seed=5)
    vpp = ctx.get_padded_velocity()
    data = np.random.default_rng(3).standard_normal((len(w.rec), w.nt)).astype(np.float32)
    ref = orc.ref_run(params, vpp, abc=False, backward=backward, adj=data, want_acc=True)
    if backward == 1:
        ctx.rtm_shots([0], data)
    else:
        ctx.gradient_shots([0], data)
    img, ill = ctx.get_accumulators()
    e_img, e_ill = rel_l2(img, ref["image"]), rel_l2(ill, ref["illum"])
    assert e_img < TOL_IMAGE and e_ill < TOL_IMAGE, f"image {e_img:.3e} illum {e_ill:.3e}"
