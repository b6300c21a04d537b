"""FWI driver over the C ABI: misfit, gradient, parabolic line search and the
learned-step accept rule.

The plain method is the reference's (src/inversion/inversion.cu:206-453):
illumination-scaled, depth-masked, -d2/dz2-filtered gradient normalised by
max|g|; parabola through the misfits of the slowness-squared steps 0,
0.02 dm and 0.05 dm (dm = 1/vmin^2 - 1/vmax^2); m <- m - step g.  This driver
uses the fixed behaviour (updated model used for the next gradient, fresh
illumination per gradient, d2/dy2 kept, source removed in the rebuild, step
bounded to [0, 8 x 0.05 dm], every model kept below the leapfrog stability
limit); inversion.exe keeps the reference's quirks for drop-in parity.

Observed, modelled and residual data stay on the GPU (torch tensors used as
device buffers); every propagation, reduction and post-processing step runs
in libfwi3d.so.  Misfits are FP64 sums of squares.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import lib
from .synth import Workload

# Largest step as a multiple of the largest trial step: the reference's parabola
# vertex is unbounded and can leave the physical range (inversion.cu:400-403).
STEP_BOUND = 8.0
# Trust region of the plain update: no cell's velocity changes by more than
# this fraction in one iteration.  The largest trial step (0.05 dm) changes
# the fastest cells of a 1500-4500 m/s model by about 15 %; a step the
# parabola extrapolates to the bound can double them, and where the clip to
# the velocity bounds catches them the model error grows while the misfit
# still falls.
MAX_DV = 0.2


@dataclass
class FwiOptions:
    batch: int = 4          # shots per launch
    zmask: float = 0.0      # depth_mask [m]
    seed: int = 1
    fixes: bool = True
    rbc: dict = field(default_factory=lambda: dict(kind=0, ratio=100.0, varVp=1000.0))


def crop(padded: np.ndarray, nb: int) -> np.ndarray:
    return np.ascontiguousarray(padded[nb:-nb, nb:-nb, nb:-nb])


def stability_velocity(dh: float, dt: float) -> float:
    """Leapfrog limit of the 8th-order 3-D stencil: v dt/dh <= 2/sqrt(3 * 6.5016)."""
    s = 2.847222222222 + 2 * (1.6 + 0.2 + 0.025396825396 + 0.001785714285)
    return 2.0 / np.sqrt(3.0 * s) * dh / dt


class Fwi:
    """One inversion problem: geometry, observed data, two library contexts."""

    def __init__(self, w: Workload, opts: FwiOptions | None = None, obs=None):
        import torch
        self.torch = torch
        self.w, self.o = w, opts or FwiOptions()
        flags = (lib.FLAG_GRAD_DY | lib.FLAG_SUBTRACT_SOURCE) if self.o.fixes else 0
        self.abc = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_ABC,
                               w.abc_factor, self.o.batch, 0)
        self.rbc = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC, 0.0,
                               self.o.batch, flags)
        for c in (self.abc, self.rbc):
            c.set_geometry(w.src, w.rec, w.rec_first, w.rec_count)
        self.nshot = len(w.src)
        counts = [self.abc.shot_nrec(s) * w.nt for s in range(self.nshot)]
        self.offset = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        n = int(self.offset[-1])
        self.cal = torch.empty(n, device="cuda", dtype=torch.float32)
        self.res = torch.empty(n, device="cuda", dtype=torch.float32)
        self.obs = obs if obs is not None else self.model(w.vp)
        self.evals = 0
        self.gradients = 0
        self.vbounds = (0.0, np.inf)

    # -- building blocks ------------------------------------------------------
    def _batches(self):
        B = self.o.batch
        return [list(range(s, min(s + B, self.nshot))) for s in range(0, self.nshot, B)]

    def model(self, v):
        """Seismograms of every shot for velocity v (device tensor)."""
        out = self.torch.empty(int(self.offset[-1]), device="cuda", dtype=self.torch.float32)
        self.abc.set_velocity(v)
        self.torch.cuda.synchronize()
        for b in self._batches():
            self.abc.model_shots_dev(b, out.data_ptr() + 4 * int(self.offset[b[0]]))
        return out

    def misfit(self, v) -> float:
        """sum (obs - cal)^2 over every shot and sample (FP64)."""
        self.abc.set_velocity(v)
        for b in self._batches():
            self.abc.model_shots_dev(b, self.cal.data_ptr() + 4 * int(self.offset[b[0]]))
        self.evals += 1
        return self.abc.residual_dev(self.obs.data_ptr(), self.cal.data_ptr(), int(self.offset[-1]),
                                     self.res.data_ptr())

    def gradient(self, v):
        """Misfit of v, then the gradient: returns (post-processed gradient,
        raw cropped gradient, cropped illumination, misfit)."""
        f = self.misfit(v)
        self.rbc.reset_accumulators()
        self.rbc.set_velocity(v)
        # the random pads depend only on how many gradients came before, so two
        # runs that take the same steps see the same pads
        for k, b in enumerate(self._batches()):
            self.rbc.apply_random_boundary(seed=self.o.seed + 7919 * self.gradients + k, **self.o.rbc)
            self.rbc.gradient_shots_dev(b, self.res.data_ptr() + 4 * int(self.offset[b[0]]))
        self.gradients += 1
        g, _ = self.rbc.gradient_post(self.o.zmask)
        raw, ill = self.rbc.get_accumulators()
        return g, crop(raw, self.w.nb), crop(ill, self.w.nb), f

    # -- plain line search ----------------------------------------------------
    def line_search(self, v, g, f0, dm):
        """Bounded parabolic step on m = 1/v^2, within the MAX_DV trust
        region.  Returns (new velocity, step, the parabola's predicted misfit
        at the step)."""
        if not (dm > 0) or not np.all(np.isfinite(g)) or not np.any(g):
            return v, 0.0, f0
        m = 1.0 / (v.astype(np.float64) ** 2)
        g64 = np.asarray(g, np.float64)
        a = np.array([0.0, 0.02 * dm, 0.05 * dm])
        lo, hi = self.vbounds

        def trial(alpha):
            # FP64 throughout, whatever the type of alpha: a Python float times
            # an FP32 array would round the product to FP32, so the same step
            # would give a slightly different model each way it is written
            return np.clip(1.0 / np.sqrt(np.maximum(m - float(alpha) * g64, 1e-12)), lo, hi).astype(np.float32)
        f = np.array([f0, self.misfit(trial(a[1])), self.misfit(trial(a[2]))])
        # the reference fits the parabola to sqrt(sum res^2) (inversion.cu:390-403)
        r = np.sqrt(f)
        num = (a[1] ** 2 - a[2] ** 2) * r[0] + (a[2] ** 2 - a[0] ** 2) * r[1] + (a[0] ** 2 - a[1] ** 2) * r[2]
        den = (a[1] - a[2]) * r[0] + (a[2] - a[0]) * r[1] + (a[0] - a[1]) * r[2]
        step = 0.5 * num / den if den != 0 else 0.0
        convex = (r[2] - r[1]) / (a[2] - a[1]) > (r[1] - r[0]) / (a[1] - a[0])
        if not convex or not step > 0:
            step = float(a[int(np.argmin(r))])
        step = min(step, STEP_BOUND * a[2])
        # the velocity change grows about linearly with the step: shrink it
        # until the largest relative change is within MAX_DV
        v64 = v.astype(np.float64)
        for _ in range(4):
            rel = float(np.max(np.abs(trial(step).astype(np.float64) / v64 - 1.0))) if step > 0 else 0.0
            if rel <= MAX_DV * (1 + 1e-6):
                break
            step *= MAX_DV / rel
        # the parabola through the trials, evaluated at the step (Lagrange form)
        lag = sum(r[i] * np.prod([(step - a[j]) / (a[i] - a[j]) for j in range(3) if j != i]) for i in range(3))
        pred = float(f[1] if step == a[1] else f[2] if step == a[2] else f[0] if step == 0 else max(lag, 0.0) ** 2)
        return trial(step), float(step), pred


def rms(v, ref) -> float:
    return float(np.sqrt(np.mean((v.astype(np.float64) - ref.astype(np.float64)) ** 2)))


def run(prob: Fwi, v0, iterations: int, learned=None, log=print):
    """Run `iterations` updates from v0.  With `learned` (a callable mapping
    (raw gradient, velocity, illumination) to a velocity update), each
    iteration also evaluates v + learned(...) and keeps it only when its misfit
    is at most the plain step's.  Returns (final velocity, history)."""
    w = prob.w
    vmin, vmax = float(v0.min()), float(v0.max())
    dm = 1.0 / vmin ** 2 - 1.0 / vmax ** 2
    # every trial and updated model stays in a physical range below the
    # leapfrog stability limit
    prob.vbounds = (0.8 * vmin, min(1.2 * vmax, 0.98 * stability_velocity(w.dh, w.dt)))
    v = v0.astype(np.float32).copy()
    hist = []
    prob.gradients = 0
    t0 = time.perf_counter()
    for it in range(iterations):
        g, raw, ill, f0 = prob.gradient(v)
        hist.append(dict(iteration=it, misfit=f0, rms=rms(v, w.vp), time=time.perf_counter() - t0))
        v_plain, step, f_plain = prob.line_search(v, g, f0, dm)
        choice = "plain"
        v_next = v_plain
        if learned is not None:
            dv = learned(raw, v, ill)
            v_l = np.clip(v + dv, *prob.vbounds).astype(np.float32)
            f_l = prob.misfit(v_l)
            if f_l <= f_plain:
                v_next, choice = v_l, "learned"
            hist[-1].update(f_learned=f_l)
        hist[-1].update(step=step, f_plain_pred=f_plain, choice=choice)
        log(f"iter {it}: misfit {f0:.6e} rms {hist[-1]['rms']:.2f} step {step:.3e} -> {choice}")
        v = v_next
    f = prob.misfit(v)
    hist.append(dict(iteration=iterations, misfit=f, rms=rms(v, w.vp), time=time.perf_counter() - t0))
    log(f"final: misfit {f:.6e} rms {hist[-1]['rms']:.2f} after {hist[-1]['time']:.1f} s")
    return v, hist
