"""Inputs of the golden fixtures, rebuilt deterministically from seeds.

The fixtures in this folder hold outputs of the reference's own CUDA kernels
(phbastosa/FWI3D built from its sources, oracle/_ref) run on a B200 by
make_golden.py.  The grid is large enough that the reference's source
injection (thread 0 of block 0 atomically adds the source while every other
block reads P, src/modeling/modeling.cu:347-348) completes before the block
that owns the source cell starts; on small grids that race makes the
reference's own output change from run to run.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import oracle as orc  # noqa: E402
from fwi3d_b200 import synth  # noqa: E402

HERE = Path(__file__).resolve().parent
ABC_FACTOR = 0.02


def workload():
    """84 x 88 x 86 layered model with a 2 % random texture, 8-cell pad,
    source in the middle of the volume, 5 x 5 receivers 30 m deep."""
    w = synth.small_case(n=84, nb=8, nt=200, seed=11)
    w.src = np.array([[w.nx * w.dh / 2, w.ny * w.dh / 2, w.nz * w.dh / 2]], np.float32)
    w.abc_factor = ABC_FACTOR
    return w


def random_pad(w, seed=21, ratio=0.3):
    """Edge-replicated model whose pad is scaled by 1 + ratio * ramp * U(-1, 1),
    ramp = depth into the pad / nb (numpy PCG64, so identical everywhere)."""
    vpp = orc.expand(w.vp, w.nz, w.nx, w.ny, w.nb).astype(np.float32)
    nyy, nxx, nzz = vpp.shape
    nb = w.nb

    def ramp(n):
        i = np.arange(n)
        d = np.where(i < nb, nb - i, np.where(i >= n - nb, i - (n - nb - 1), 0))
        return d / nb

    r = np.maximum(np.maximum(ramp(nyy)[:, None, None], ramp(nxx)[None, :, None]), ramp(nzz)[None, None, :])
    u = np.random.default_rng(seed).uniform(-1, 1, vpp.shape)
    return (vpp * (1 + ratio * r * u)).astype(np.float32)


def adjoint_data(w, seed=3):
    return np.random.default_rng(seed).standard_normal((len(w.rec), w.nt)).astype(np.float32)


def slices(vol):
    """Three orthogonal planes through the middle of a padded volume."""
    nyy, nxx, nzz = vol.shape
    return [np.ascontiguousarray(vol[nyy // 2]), np.ascontiguousarray(vol[:, nxx // 2]),
            np.ascontiguousarray(vol[:, :, nzz // 2])]


def load(name):
    return np.load(HERE / f"{name}.npz")
