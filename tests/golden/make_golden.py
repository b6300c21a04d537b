"""Generate the golden fixtures from the reference's own CUDA build.

Needs a GPU and oracle/_ref/libref_fwi3d.so (built by `make -C oracle ref`
from the reference sources).  Writes, in this folder:
  ref_abc_forward.npz   seismogram of Modeling::forward_solver with the Cerjan sponge
  ref_rbc_rtm.npz       seismogram, image and illumination slices (migration kernels)
  ref_rbc_gradient.npz  gradient and illumination slices (inversion kernels)
Each fixture also stores the reference run-to-run spread (two runs).

    python tests/golden/make_golden.py
"""
import json
import tempfile

import numpy as np

import golden_cases as gc
import oracle as orc


def main():
    w = gc.workload()
    tmp = tempfile.mkdtemp()
    params = orc.write_reference_setup(tmp, w.nz, w.nx, w.ny, w.dh, w.nt, w.dt, w.fmax, w.nb, w.src, w.rec,
                                       abc_factor=gc.ABC_FACTOR)
    meta = dict(nz=w.nz, nx=w.nx, ny=w.ny, nb=w.nb, dh=w.dh, nt=w.nt, dt=w.dt, fmax=w.fmax,
                abc_factor=gc.ABC_FACTOR, source=w.src.tolist())

    vpp = orc.expand(w.vp, w.nz, w.nx, w.ny, w.nb).astype(np.float32)
    a = orc.ref_run(params, vpp, abc=True)
    b = orc.ref_run(params, vpp, abc=True)
    spread = float(np.linalg.norm(a["seis"] - b["seis"]) / np.linalg.norm(a["seis"]))
    np.savez_compressed(gc.HERE / "ref_abc_forward.npz", seis=a["seis"], tlag=a["tlag"], spread=spread,
                        meta=json.dumps(meta))
    print("abc forward: run-to-run", spread)

    vpr = gc.random_pad(w)
    data = gc.adjoint_data(w)
    for backward, name in ((1, "ref_rbc_rtm"), (2, "ref_rbc_gradient")):
        a = orc.ref_run(params, vpr, abc=False, backward=backward, adj=data, want_acc=True)
        b = orc.ref_run(params, vpr, abc=False, backward=backward, adj=data, want_acc=True)
        spread = float(np.linalg.norm(a["image"] - b["image"]) / np.linalg.norm(a["image"]))
        out = dict(seis=a["seis"], tlag=a["tlag"], spread=spread, meta=json.dumps(meta),
                   image_norm=np.linalg.norm(a["image"].astype(np.float64)),
                   illum_norm=np.linalg.norm(a["illum"].astype(np.float64)))
        for k, s in enumerate(gc.slices(a["image"])):
            out[f"image{k}"] = s
        for k, s in enumerate(gc.slices(a["illum"])):
            out[f"illum{k}"] = s
        np.savez_compressed(gc.HERE / f"{name}.npz", **out)
        print(name, "run-to-run", spread)


if __name__ == "__main__":
    main()
