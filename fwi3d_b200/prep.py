"""Pipeline preparation around the hot path, file-compatible with the
reference's helper scripts:

    python -m fwi3d_b200.prep setup parameters.txt
        acquisition grid and start model (run/generate_setup.py:24-68): a 6 x 6
        shot grid over 1000-4000 m at 100 m depth and 51 x 51 receivers over
        0-5000 m at the surface, written as "%.2f" CSV to the SPS/RPS files;
        start model 1 / gaussian_filter(1 / v_true, 3 cells) with the true model
        kept above depth_mask, written next to model_file with "true" replaced
        by "init"
    python -m fwi3d_b200.prep input-data parameters.txt [--folder DIR]
        RTM input gathers (run/generate_input_data.py:28-46) on the GPU through
        fwi_prepare_rtm_input: every seismogram_nt{nt}_nr{nr}_{us}us_shot_{s}.bin
        in DIR (default: mod_output_folder) becomes input_RTM_seismogram_...bin

Both read parameters.txt through the reference's own lookup rule
(fwi_catch_parameter).
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

from . import lib


def _p(params, key):
    return lib.catch_parameter(params, key)


def setup(params) -> None:
    from scipy.ndimage import gaussian_filter
    nx, ny, nz = (int(_p(params, k)) for k in ("x_samples", "y_samples", "z_samples"))
    dh = float(_p(params, "model_spacing"))
    nsx = nsy = 6
    nrx = nry = 51
    sx, sy = np.meshgrid(np.linspace(1000, 4000, nsx), np.linspace(1000, 4000, nsy))
    rx, ry = np.meshgrid(np.linspace(0, 5000, nrx), np.linspace(0, 5000, nry))
    sps = np.zeros((nsx * nsy, 3))
    rps = np.zeros((nrx * nry, 3))
    sps[:, 0] = sx.reshape(-1, order="F")
    sps[:, 1] = sy.reshape(-1, order="F")
    sps[:, 2] = 100.0
    rps[:, 0] = rx.reshape(-1, order="F")
    rps[:, 1] = ry.reshape(-1, order="F")
    np.savetxt(_p(params, "SPS"), sps, fmt="%.2f", delimiter=",")
    np.savetxt(_p(params, "RPS"), rps, fmt="%.2f", delimiter=",")
    model_file = _p(params, "model_file")
    m_true = np.fromfile(model_file, dtype=np.float32, count=nx * ny * nz).reshape([nz, nx, ny], order="F")
    m_init = 1.0 / gaussian_filter(1.0 / m_true, 3.0)
    zid = int(float(_p(params, "depth_mask")) / dh)
    m_init[:zid] = m_true[:zid]
    m_init.flatten("F").astype(np.float32).tofile(model_file.replace("true", "init"))


def input_data(params, folder=None, velocity=3600.0, time_delay=0.18, gstd=30.0) -> list[Path]:
    nt = int(_p(params, "time_samples"))
    dt = float(_p(params, "time_spacing"))
    sps = lib.read_points(_p(params, "SPS"))
    rps = lib.read_points(_p(params, "RPS"))
    folder = Path(folder or _p(params, "mod_output_folder"))
    out = []
    for s in range(len(sps)):
        name = f"seismogram_nt{nt}_nr{len(rps)}_{dt * 1e6:.0f}us_shot_{s + 1}.bin"
        d = np.fromfile(folder / name, np.float32, count=nt * len(rps)).reshape(len(rps), nt)
        m = lib.prepare_rtm_input(d, rps, sps[s], np.float32(dt), velocity, time_delay, gstd)
        dst = folder / ("input_RTM_" + name)
        m.tofile(dst)
        out.append(dst)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("setup")
    s.add_argument("parameters")
    i = sub.add_parser("input-data")
    i.add_argument("parameters")
    i.add_argument("--folder", default=None)
    a = ap.parse_args(argv)
    if a.cmd == "setup":
        setup(a.parameters)
    else:
        for f in input_data(a.parameters, a.folder):
            print(f)


if __name__ == "__main__":
    main(sys.argv[1:])
