"""Parity cases shared by the GPU tests: one small workload run through the
CUDA library and through the FP64 oracle on identical inputs."""
from __future__ import annotations

import numpy as np

import oracle as orc
from fwi3d_b200 import lib, synth

# Tolerances (relative L2 error of the FP32 CUDA path against the FP64 oracle).
# The stencil, the wavefields and the accumulators are FP32; the oracle is FP64
# throughout.
TOL_SEIS = 2e-5
TOL_IMAGE = 2e-4
TOL_GRAD = 2e-4


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def interior(a, nb: int) -> np.ndarray:
    """The physical box of a padded volume: by default the library accumulates
    images, gradients and illumination there only (the reference's
    post-processing crops the pad away before it reads them)."""
    return np.asarray(a)[nb:-nb, nb:-nb, nb:-nb]


def indices(w: synth.Workload, nb: int):
    """Flat padded indices of the source(s) and receivers (oracle mapping)."""
    nzz, nxx = w.nz + 2 * nb, w.nx + 2 * nb

    def flat(p):
        i = orc.grid_index(float(p[2]), w.dh, nb)
        j = orc.grid_index(float(p[0]), w.dh, nb)
        k = orc.grid_index(float(p[1]), w.dh, nb)
        return orc.flat_index(i, j, k, nzz, nxx)

    return [flat(s) for s in w.src], np.array([flat(r) for r in w.rec], np.int64)


def context(w: synth.Workload, boundary, max_batch=1, flags=0, abc_factor=None):
    ctx = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, boundary,
                      w.abc_factor if abc_factor is None else abc_factor, max_batch, flags)
    ctx.set_geometry(w.src, w.rec, w.rec_first, w.rec_count)
    return ctx


def oracle_wavelet(ctx: lib.Context, w: synth.Workload):
    """The FP32 host wavelet the library uses (reference formula) as FP64,
    so that both sides inject the same source samples."""
    wf, tl = orc.wavelet(w.nt, w.dt, w.fmax)
    assert tl == ctx.tlag
    # the library evaluates the reference's FP32 host formula; reproduce it
    pi = np.float32(np.pi)
    t0 = np.float32(2.0) * np.sqrt(pi) / np.float32(w.fmax)
    fc = np.float32(w.fmax) / (np.float32(3.0) * np.sqrt(pi))
    n = np.arange(w.nt, dtype=np.float32)
    td = n * np.float32(w.dt) - t0
    arg = pi * pi * pi * fc * fc * td * td
    w32 = np.float32(1e5) * (np.float32(1.0) - np.float32(2.0) * arg) * np.exp(-arg)
    return w32.astype(np.float64), wf
