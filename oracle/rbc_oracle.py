"""NumPy restatement of the random-boundary pad -- TEST INFRASTRUCTURE ONLY.

The checker for fwi_apply_random_boundary (rbc_background_kernel and
rbc_blobs_kernel in fwi3d_b200/csrc/aux_kernels.cuh); only tests/ use it.

The recipe is the reference's set_random_boundary (phbastosa/FWI3D,
src/modeling/modeling.cu:558-673):

  background (random_boundary_bg, :617-666): every cell outside the index box
      [nb, n - nb) on all axes starts from the nearest model-edge value and,
      for every axis a on which it lies in the pad, adds
      (1 - depth_a / nb) * varVp * N(0, 1), in the order x, y, z;
  blobs (random_boundary_gp, :594-615, placed by :566-591): Poisson-disk
      points outside the inner half-pad box, each a Gaussian
      +-A exp(-|x - c|^2 / (2 r^2)) added to every cell outside the physical
      box (nb dh, max - nb dh) and followed by the clamp
      [vmin - varVp, vmax + varVp].

The reference draws its normals from cuRAND seeded with clock64() (:668-673);
the library draws them from a counter-based hash of (seed, stream, cell): the
SplitMix64 output function of Steele, Lea and Flood (OOPSLA 2014), the top 24
bits as a uniform in (0, 1), Box-Muller in FP64 rounded once to FP32.  Every
FP32 product and sum is rounded on its own on the device, so the background
below is the same FP32 arithmetic and must match bit for bit.  The blob pass
uses expf on the device and exp here, so it matches to a few FP32 ulps.

Volumes are numpy (nyy, nxx, nzz) float32 (z fastest).
"""
from __future__ import annotations

import numpy as np

F32 = np.float32
_C1 = np.uint64(0x9E3779B97F4A7C15)
_C2 = np.uint64(0xBF58476D1CE4E5B9)
_C3 = np.uint64(0x94D049BB133111EB)
_CS = np.uint64(0x632BE59BD9B4E019)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 output function on uint64 arrays (wrapping arithmetic)."""
    x = np.asarray(x, np.uint64)
    with np.errstate(over="ignore"):
        x = x + _C1
        x = (x ^ (x >> np.uint64(30))) * _C2
        x = (x ^ (x >> np.uint64(27))) * _C3
    return x ^ (x >> np.uint64(31))


def uniform01(seed: int, stream: int, ctr: np.ndarray) -> np.ndarray:
    """(top 24 bits + 0.5) / 2^24 as FP32: exact in FP32."""
    ctr = np.asarray(ctr, np.uint64)
    with np.errstate(over="ignore"):
        inner = splitmix64(np.uint64(stream) * _CS + ctr)
    h = splitmix64(np.uint64(seed) ^ inner)
    return ((h >> np.uint64(40)).astype(F32) + F32(0.5)) * F32(1.0 / 16777216.0)


def normal01(seed: int, stream: int, ctr: np.ndarray) -> np.ndarray:
    ctr = np.asarray(ctr, np.uint64)
    u1 = uniform01(seed, stream, ctr * np.uint64(2)).astype(np.float64)
    u2 = uniform01(seed, stream, ctr * np.uint64(2) + np.uint64(1)).astype(np.float64)
    return (np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)).astype(F32)


def _pad_depth(idx: np.ndarray, n: int, nb: int) -> np.ndarray:
    return np.where(idx < nb, idx, np.where(idx >= n - nb, n - 1 - idx, -1))


def background(vclean: np.ndarray, nb: int, kind: int, ratio: float, varVp: float, vlo: float, vhi: float,
               seed: int) -> np.ndarray:
    """The pad after the background pass (interior cells unchanged)."""
    v = np.array(vclean, F32, copy=True)
    nyy, nxx, nzz = v.shape
    K, J, I = np.meshgrid(np.arange(nyy), np.arange(nxx), np.arange(nzz), indexing="ij")
    inside = (I >= nb) & (I < nzz - nb) & (J >= nb) & (J < nxx - nb) & (K >= nb) & (K < nyy - nb)
    sel = ~inside
    i, j, k = I[sel], J[sel], K[sel]
    ii = np.clip(i, nb, nzz - nb - 1)
    jj = np.clip(j, nb, nxx - nb - 1)
    kk = np.clip(k, nb, nyy - nb - 1)
    val = vclean[kk, jj, ii].astype(F32)
    dz, dx, dy = _pad_depth(i, nzz, nb), _pad_depth(j, nxx, nb), _pad_depth(k, nyy, nb)
    cell = i.astype(np.uint64) + np.uint64(nzz) * (j.astype(np.uint64) + np.uint64(nxx) * k.astype(np.uint64))
    fnb = F32(nb)
    ramp = lambda d: F32(1.0) - d.astype(F32) / fnb
    if kind == 0:
        for d, stream in ((dx, 1), (dy, 2), (dz, 3)):
            m = d >= 0
            if m.any():
                t = (ramp(d[m]) * F32(varVp)) * normal01(seed, stream, cell[m])
                val[m] = val[m] + t
    else:
        r = np.zeros(val.shape, F32)
        for d in (dx, dy, dz):
            m = d >= 0
            r[m] = np.maximum(r[m], ramp(d[m]))
        u = F32(2.0) * uniform01(seed, 4, cell) - F32(1.0)
        val = val * (F32(1.0) + (F32(ratio) * r) * u)
    v[sel] = np.minimum(np.maximum(val, F32(vlo)), F32(vhi))
    return v


def blob_pass(v: np.ndarray, nb: int, dh: float, blobs: np.ndarray, vlo: float, vhi: float) -> np.ndarray:
    """Add the blobs (n, 5: x, y, z, r, signed amplitude) in order to every
    cell outside the physical inner box, each followed by the clamp; blobs are
    truncated at 5 r as on the device."""
    v = np.array(v, F32, copy=True)
    nyy, nxx, nzz = v.shape
    dh = F32(dh)
    X = np.arange(nxx, dtype=F32) * dh
    Y = np.arange(nyy, dtype=F32) * dh
    Z = np.arange(nzz, dtype=F32) * dh
    fnb = F32(nb) * dh
    xmax, ymax, zmax = F32(nxx - 1) * dh, F32(nyy - 1) * dh, F32(nzz - 1) * dh
    for bx, by, bz, r, amp in np.asarray(blobs, F32):
        ir = F32(1.0) / r
        reach = 5.0 * float(r) / float(dh) + 2
        lo = lambda c, n: max(0, int(np.floor(float(c) / float(dh) - reach)))
        hi = lambda c, n: min(n, int(np.ceil(float(c) / float(dh) + reach)) + 1)
        ks, js, is_ = slice(lo(by, nyy), hi(by, nyy)), slice(lo(bx, nxx), hi(bx, nxx)), slice(lo(bz, nzz), hi(bz, nzz))
        ex = (X[js] - bx) * ir
        ey = (Y[ks] - by) * ir
        ez = (Z[is_] - bz) * ir
        e2 = ex[None, :, None] * ex[None, :, None] + ey[:, None, None] * ey[:, None, None] + ez[None, None, :] * ez[None, None, :]
        outside = ~((X[js][None, :, None] > fnb) & (X[js][None, :, None] < xmax - fnb)
                    & (Y[ks][:, None, None] > fnb) & (Y[ks][:, None, None] < ymax - fnb)
                    & (Z[is_][None, None, :] > fnb) & (Z[is_][None, None, :] < zmax - fnb))
        m = outside & (e2 <= F32(25.0))
        sub = v[ks, js, is_]
        add = amp * np.exp(F32(-0.5) * e2).astype(F32)
        sub = np.where(m, np.minimum(np.maximum(sub + add, F32(vlo)), F32(vhi)), sub)
        v[ks, js, is_] = sub
    return v
