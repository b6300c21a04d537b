"""FP32-vs-FP64 accuracy of the mixed-precision gradient workload (401 x 401 x
201 model at 12.5 m, 41-cell pad: 483 x 483 x 283 padded cells), measured
against the FP64 oracle on the full grid with a shortened time axis and one
shot (the oracle needs minutes per sweep at this size).

Reports the relative L2 error of the seismogram (Cerjan modeling), of the raw
gradient and illumination (random-boundary fused pass), of the post-processed
gradient and of the parabolic line-search step (FP32 propagation + FP64
misfit sums on the GPU against FP64 everywhere).

With the shortened time axis the source field reaches only part of the
model; elsewhere gradient / illumination is noise over noise (FP32 flushes
it to exact zeros, FP64 does not), and max|g| would normalise by that noise.
The post-processed gradient and the step are therefore compared over the
illuminated cells (illumination >= 1e-3 of its maximum on the oracle side),
with each side's unnormalised gradient renormalised there.  Run on a GPU box:

    python tests/accuracy_report.py [--nt 300] [--out report.json]
"""
import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent / "oracle"))
sys.path.insert(0, str(HERE))

import oracle as orc  # noqa: E402
from cases import indices, oracle_wavelet, rel_l2  # noqa: E402
from fwi3d_b200 import lib, synth  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nt", type=int, default=300)
    ap.add_argument("--shot", type=int, default=5)
    ap.add_argument("--out", default="")
    a = ap.parse_args()
    t0 = time.perf_counter()
    w = synth.gradient_401(nt=a.nt)
    s = a.shot
    w.src = w.src[s:s + 1]
    rep = {"workload": w.name, "nt": a.nt, "shot": s, "oracle_threads": orc.num_threads()}

    # Cerjan modeling: observed (true model) and calculated (start model)
    abc = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_ABC, w.abc_factor)
    abc.set_geometry(w.src, w.rec)
    w64, _ = oracle_wavelet(abc, w)
    src, rec = indices(w, w.nb)
    seis = {}
    for name, v in (("obs", w.vp), ("cal", w.start)):
        abc.set_velocity(v)
        g = abc.model_shots([0])[0]
        vpp = abc.get_padded_velocity()
        o, _, _ = orc.forward(vpp, w.dh, w.dt, w.nt, abc.tlag, w64, src[0], rec, abc=True, nb=w.nb,
                              factor=w.abc_factor)
        seis[name] = (g, o)
        rep[f"seismogram_{name}_rel_l2"] = rel_l2(g, o)
    res_g = (seis["obs"][0] - seis["cal"][0]).astype(np.float32)
    res_o = seis["obs"][1] - seis["cal"][1]
    rep["misfit_rel_err"] = abs(float(np.sum(res_g.astype(np.float64) ** 2)) / float(np.sum(res_o ** 2)) - 1)
    print(f"modeling done {time.perf_counter() - t0:.0f} s", flush=True)

    # gradient through one random boundary, same residual on both sides
    rbc = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC)
    rbc.set_geometry(w.src, w.rec)
    rbc.set_velocity(w.start)
    rbc.apply_random_boundary(seed=3, **w.rbc)
    vpr = rbc.get_padded_velocity()
    rbc.gradient_shots([0], res_g)
    graw, gill = rbc.get_accumulators()
    gpost, gmax = rbc.gradient_post(w.zmask)
    _, P, Q = orc.forward(vpr, w.dh, w.dt, w.nt, rbc.tlag, w64, src[0], rec)
    oimg, oill, _, _ = orc.backward(vpr, w.dh, w.dt, w.nt, rbc.tlag, rec, res_g, P, Q, mode=1)
    del P, Q
    opost, omax = orc.gradient_post(oimg, oill, w.nz, w.nx, w.ny, w.nb, w.dh, w.zmask)
    rep["gradient_raw_rel_l2"] = rel_l2(graw, oimg)
    rep["illumination_rel_l2"] = rel_l2(gill, oill)
    ill_c = orc.reduce(oill, w.nz, w.nx, w.ny, w.nb)
    lit = ill_c >= 1e-3 * ill_c.max()
    rep["illuminated_fraction"] = float(lit.mean())
    gu = np.where(lit, gpost.astype(np.float64) * gmax, 0.0)
    ou = np.where(lit, opost * omax, 0.0)
    gpost = gu / np.abs(gu).max()
    opost = ou / np.abs(ou).max()
    rep["gradient_post_rel_l2"] = rel_l2(gpost, opost)
    print(f"gradient done {time.perf_counter() - t0:.0f} s", flush=True)

    # parabolic step on slowness squared from both gradients
    dm = 1.0 / float(w.start.min()) ** 2 - 1.0 / float(w.start.max()) ** 2
    a_tr = [0.0, 0.02 * dm, 0.05 * dm]
    m = 1.0 / w.start.astype(np.float64) ** 2
    obs_g, obs_o = seis["obs"]
    fg, fo = [], []
    for alpha in a_tr:
        vg = (1.0 / np.sqrt(m - alpha * gpost.astype(np.float64))).astype(np.float32)
        vo = 1.0 / np.sqrt(m - alpha * opost)
        abc.set_velocity(vg)
        cal = abc.model_shots([0])[0]
        fg.append(float(np.sum((obs_g - cal).astype(np.float64) ** 2)))
        vpo = orc.expand(vo, w.nz, w.nx, w.ny, w.nb)
        oc, _, _ = orc.forward(vpo, w.dh, w.dt, w.nt, abc.tlag, w64, src[0], rec, abc=True, nb=w.nb,
                               factor=w.abc_factor)
        fo.append(float(np.sum((obs_o - oc) ** 2)))
    sg = orc.parabola_step(*a_tr, *np.sqrt(fg))
    so = orc.parabola_step(*a_tr, *np.sqrt(fo))
    rep["misfits_gpu"], rep["misfits_oracle"] = fg, fo
    rep["step_gpu"], rep["step_oracle"] = sg, so
    rep["step_rel_err"] = abs(sg / so - 1)
    rep["seconds"] = time.perf_counter() - t0
    print(json.dumps(rep, indent=1), flush=True)
    if a.out:
        Path(a.out).write_text(json.dumps(rep, indent=1))


if __name__ == "__main__":
    main()
