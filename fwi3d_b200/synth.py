"""Seeded synthetic models and acquisition geometries.

The reference ships no input model (its overthrust model is absent) and no
benchmark data set; these generators build the five workloads the project is
measured on (layered models, Gaussian anomalies, surface shot/receiver grids)
in the reference's layouts.  Volumes are float32 C-order (ny, nx, nz), z
fastest; coordinates are metres (x, y, z).

The smoothed start models follow run/generate_setup.py:64 (smoothing in
slowness: 1 / gaussian(1 / v)).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def layered(nz, nx, ny, dh, velocities, tops=None, dips_deg=None, azimuths_deg=None):
    """Velocity model of stacked layers.  tops[k] is the depth [m] of the top
    of layer k at the model centre (tops[0] = 0); a dipping interface rises or
    falls by tan(dip) along its azimuth."""
    n = len(velocities)
    if tops is None:
        tops = np.arange(n) * (nz * dh / n)
    tops = np.asarray(tops, float)
    dips = np.zeros(n) if dips_deg is None else np.radians(np.asarray(dips_deg, float))
    az = np.zeros(n) if azimuths_deg is None else np.radians(np.asarray(azimuths_deg, float))
    z = np.arange(nz) * dh
    x = (np.arange(nx) - (nx - 1) / 2) * dh
    y = (np.arange(ny) - (ny - 1) / 2) * dh
    Y, X, Z = np.meshgrid(y, x, z, indexing="ij")
    v = np.full((ny, nx, nz), velocities[0], np.float64)
    for k in range(1, n):
        depth = tops[k] + np.tan(dips[k]) * (X * np.cos(az[k]) + Y * np.sin(az[k]))
        v = np.where(Z >= depth, velocities[k], v)
    return v.astype(np.float32)


def add_gaussian(v, dh, centre_xyz, sigma, rel):
    """Multiply v by 1 + rel * exp(-|r - c|^2 / (2 sigma^2))."""
    ny, nx, nz = v.shape
    z = np.arange(nz) * dh - centre_xyz[2]
    x = np.arange(nx) * dh - centre_xyz[0]
    y = np.arange(ny) * dh - centre_xyz[1]
    g = np.exp(-(y[:, None, None] ** 2 + x[None, :, None] ** 2 + z[None, None, :] ** 2) / (2 * sigma ** 2))
    return (v * (1.0 + rel * g)).astype(np.float32)


def smooth_slowness(v, sigma_m, dh):
    """Start model 1 / gaussian_filter(1 / v, sigma) as in run/generate_setup.py:64."""
    from scipy.ndimage import gaussian_filter
    return (1.0 / gaussian_filter(1.0 / v.astype(np.float64), sigma_m / dh)).astype(np.float32)


def surface_grid(xs, ys, z):
    """All (x, y, z) combinations, x fastest (the SPS/RPS order of
    run/generate_setup.py:42-48)."""
    X, Y = np.meshgrid(np.asarray(xs, float), np.asarray(ys, float))
    return np.stack([X.ravel(), Y.ravel(), np.full(X.size, float(z))], axis=1).astype(np.float32)


@dataclass
class Workload:
    name: str
    nz: int
    nx: int
    ny: int
    dh: float
    nt: int
    dt: float
    fmax: float
    nb: int
    vp: np.ndarray
    src: np.ndarray
    rec: np.ndarray
    rec_first: np.ndarray | None = None
    rec_count: np.ndarray | None = None
    start: np.ndarray | None = None
    rbc: dict = field(default_factory=dict)
    abc_factor: float = 0.004
    zmask: float = 0.0  # depth_mask [m]: gradient muted above it (acquisition imprint)


def modeling_101(nt=1001):
    """Plain single-shot modeling: 101^3 at 10 m, four flat layers
    1500/2000/2700/3500 m/s, 50-cell random pad (+-40 % uniform, ramped with
    depth into the pad), Ricker 10 Hz peak at the centre, 10 m deep, 51 x 51
    receivers every 20 m at 10 m depth."""
    n, dh = 101, 10.0
    v = layered(n, n, n, dh, [1500, 2000, 2700, 3500])
    src = np.array([[500.0, 500.0, 10.0]], np.float32)
    rec = surface_grid(np.arange(51) * 20.0, np.arange(51) * 20.0, 10.0)
    return Workload("modeling-101^3", n, n, n, dh, nt, 1e-3, 30.0, 50, v, src, rec,
                    rbc=dict(kind=1, ratio=0.4, varVp=0.0))


def rtm_201(nt=2001, nshots=64, seed=2):
    """Batched RTM: 201^3 at 10 m, five layers plus Gaussian anomalies of -8 %
    and +12 % (sigma 150 m); migration model smoothed with sigma 200 m; 64 shots
    on an 8 x 8 grid, each with its own 121 x 121 receiver patch (10 m) clipped
    to the model."""
    n, dh = 201, 10.0
    v = layered(n, n, n, dh, [1500, 1800, 2200, 2600, 3000], tops=[0, 300, 700, 1100, 1500])
    v = add_gaussian(v, dh, (700.0, 800.0, 900.0), 150.0, -0.08)
    v = add_gaussian(v, dh, (1300.0, 1200.0, 1300.0), 150.0, +0.12)
    side = int(round(np.sqrt(nshots)))
    centres = (np.arange(side) + 0.5) * (2000.0 / side)
    src = surface_grid(centres, centres, 10.0)[:nshots]
    recs, first, count = [], [], []
    for s in src:
        xs = s[0] + (np.arange(121) - 60) * 10.0
        ys = s[1] + (np.arange(121) - 60) * 10.0
        xs = xs[(xs >= 0) & (xs <= (n - 1) * dh)]
        ys = ys[(ys >= 0) & (ys <= (n - 1) * dh)]
        r = surface_grid(xs, ys, 10.0)
        first.append(sum(len(q) for q in recs))
        count.append(len(r))
        recs.append(r)
    start = smooth_slowness(v, 200.0, dh)
    return Workload("rtm-201^3-64shots", n, n, n, dh, nt, 1e-3, 30.0, 50, v, src, np.concatenate(recs),
                    np.array(first, np.int32), np.array(count, np.int32), start=start,
                    rbc=dict(kind=0, ratio=100.0, varVp=1000.0))


def gradient_401(nt=2501, seed=3):
    """Mixed-precision gradient: 401 x 401 x 201 at 12.5 m, 8 random layers with
    velocities U(1500, 4000) and interfaces dipping up to 10 degrees, 16 shots on
    a 4 x 4 grid, a full surface spread every 25 m."""
    rng = np.random.default_rng(seed)
    nz, nx, ny, dh = 201, 401, 401, 12.5
    vels = np.sort(rng.uniform(1500, 4000, 8))
    tops = np.concatenate([[0.0], np.sort(rng.uniform(0.1, 0.9, 7)) * nz * dh])
    v = layered(nz, nx, ny, dh, vels, tops, rng.uniform(0, 10, 8), rng.uniform(0, 360, 8))
    xs = (np.arange(4) + 0.5) * (nx - 1) * dh / 4
    src = surface_grid(xs, xs, 12.5)
    rec = surface_grid(np.arange(0, (nx - 1) * dh + 1e-3, 25.0), np.arange(0, (ny - 1) * dh + 1e-3, 25.0), 12.5)
    return Workload("gradient-401x401x201", nz, nx, ny, dh, nt, 1e-3, 30.0, 41, v, src, rec,
                    start=smooth_slowness(v, 200.0, dh), rbc=dict(kind=0, ratio=100.0, varVp=1000.0),
                    zmask=100.0)


def cnn_128(index, nt=1201):
    """Learned-preconditioner training model `index`: 128^3 at 10 m, 6 layers
    with 1-4 Gaussian anomalies of +-15 % (sigma 80-250 m); start model smoothed
    with sigma 150 m; 9 shots on a 3 x 3 grid."""
    rng = np.random.default_rng(1000 + index)
    n, dh = 128, 10.0
    vels = np.sort(rng.uniform(1500, 3500, 6))
    tops = np.concatenate([[0.0], np.sort(rng.uniform(0.08, 0.92, 5)) * n * dh])
    v = layered(n, n, n, dh, vels, tops)
    for _ in range(rng.integers(1, 5)):
        c = rng.uniform(0.2, 0.8, 3) * (n - 1) * dh
        v = add_gaussian(v, dh, c, rng.uniform(80, 250), rng.choice([-0.15, 0.15]))
    xs = (np.arange(3) + 0.5) * (n - 1) * dh / 3
    src = surface_grid(xs, xs, 10.0)
    rec = surface_grid(np.arange(0, (n - 1) * dh + 1e-3, 20.0), np.arange(0, (n - 1) * dh + 1e-3, 20.0), 10.0)
    return Workload(f"cnn-128^3-{index}", n, n, n, dh, nt, 1e-3, 30.0, 50, v, src, rec,
                    start=smooth_slowness(v, 150.0, dh), rbc=dict(kind=0, ratio=100.0, varVp=1000.0),
                    zmask=60.0)


def fwi_301(nt=2001):
    """Full FWI comparison: 301 x 301 x 151 at 10 m, layered background plus
    three +-10 % anomalies (sigma 200 m), start model smoothed with sigma 200 m,
    36 shots on a 6 x 6 grid, receivers every 20 m, 8 Hz Ricker peak."""
    nz, nx, ny, dh = 151, 301, 301, 10.0
    v = layered(nz, nx, ny, dh, [1500, 1900, 2400, 2900, 3400], tops=[0, 250, 550, 900, 1250])
    for c, a in (((900.0, 1000.0, 700.0), 0.10), ((2000.0, 1800.0, 800.0), -0.10), ((1500.0, 2200.0, 1100.0), 0.10)):
        v = add_gaussian(v, dh, c, 200.0, a)
    xs = (np.arange(6) + 0.5) * (nx - 1) * dh / 6
    src = surface_grid(xs, xs, 10.0)
    rec = surface_grid(np.arange(0, (nx - 1) * dh + 1e-3, 20.0), np.arange(0, (ny - 1) * dh + 1e-3, 20.0), 10.0)
    return Workload("fwi-301x301x151", nz, nx, ny, dh, nt, 1e-3, 24.0, 50, v, src, rec,
                    start=smooth_slowness(v, 200.0, dh), rbc=dict(kind=0, ratio=100.0, varVp=1000.0),
                    zmask=80.0)


def small_case(n=40, nb=8, nt=120, seed=0, dh=10.0, nrec_side=5):
    """A small layered case for parity tests (seconds on the oracle)."""
    rng = np.random.default_rng(seed)
    v = layered(n, n + 4, n + 2, dh, [1500, 2000, 2600], tops=[0, n * dh / 3, 2 * n * dh / 3])
    v = add_gaussian(v, dh, (n * dh / 2, n * dh / 2, n * dh / 2), 4 * dh, 0.1)
    v = (v * (1 + 0.02 * rng.standard_normal(v.shape))).astype(np.float32)
    src = np.array([[(n + 4) * dh / 2 - 3.0, (n + 2) * dh / 2 + 4.0, 2 * dh]], np.float32)
    xs = np.linspace(2 * dh, (n + 1) * dh, nrec_side)
    rec = surface_grid(xs, np.linspace(2 * dh, n * dh, nrec_side), 3 * dh)
    return Workload(f"small-{n}", n, n + 4, n + 2, dh, nt, 1e-3, 60.0, nb, v, src, rec)


def small_fwi(index, n=48, nt=400):
    """Small inversion problem `index` for tests: n^3 at 10 m, three layers with
    one or two Gaussian anomalies of +-15 % (sigma 50-90 m), start model
    smoothed with sigma 80 m, 2 x 2 shots, receivers every 20 m, 10 Hz peak."""
    rng = np.random.default_rng(5000 + index)
    dh = 10.0
    vels = np.sort(rng.uniform(1600, 3000, 3))
    tops = [0.0, *np.sort(rng.uniform(0.25, 0.75, 2)) * n * dh]
    v = layered(n, n, n, dh, vels, tops)
    for _ in range(rng.integers(1, 3)):
        c = rng.uniform(0.3, 0.7, 3) * (n - 1) * dh
        v = add_gaussian(v, dh, c, rng.uniform(50, 90), rng.choice([-0.15, 0.15]))
    xs = (np.arange(2) + 0.5) * (n - 1) * dh / 2
    src = surface_grid(xs, xs, 10.0)
    g = np.arange(0, (n - 1) * dh + 1e-3, 20.0)
    rec = surface_grid(g, g, 10.0)
    return Workload(f"small-fwi-{index}", n, n, n, dh, nt, 1e-3, 30.0, 20, v, src, rec,
                    start=smooth_slowness(v, 80.0, dh), rbc=dict(kind=0, ratio=40.0, varVp=400.0), zmask=40.0)
