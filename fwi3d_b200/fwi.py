"""FWI driver over the C ABI: misfit, gradient, line search and the
learned-step accept rule, shot-parallel over ranks.

The plain method is the reference's (src/inversion/inversion.cu:115-362):
illumination-scaled, depth-masked, -d2/dz2-filtered gradient normalised by
max|g|, a step on the slowness-squared model m = 1/v^2 with trial steps
0.02 dm and 0.05 dm (dm = 1/vmin^2 - 1/vmax^2) and a parabola through the
square roots of the misfits, then m <- m - step g.  This driver keeps the
fixed behaviour (updated model used for the next gradient, fresh
illumination per gradient, d2/dy2 kept, source removed in the rebuild, a new
random boundary per shot) and makes the step search measured:

  - every candidate step's misfit is computed, never predicted;
  - while the misfit still falls at the largest step tried, the step doubles
    (the reference stops at its two trials and extrapolates the parabola
    without bound, inversion.cu:291-313);
  - the parabola's vertex through the best step and its neighbours is then
    measured too, and the best measured candidate is taken;
  - every step stays within STEP_BOUND x 0.05 dm and the MAX_DV trust region,
    and every model below the leapfrog stability limit.

inversion.exe keeps the reference's quirks for drop-in parity.

Shots are dealt to ranks (torch.distributed; one process per GPU): each rank
models and back-propagates its own shots, the FP64 misfit is summed over
ranks, and the padded gradient and illumination are summed before the
post-processing, so every rank takes the same steps.

Observed, modelled and residual data stay on the GPU (torch tensors used as
device buffers); every propagation, reduction and post-processing step runs
in libfwi3d.so.  Misfits are FP64 sums of squares.
"""
from __future__ import annotations

import hashlib
import time
from dataclasses import dataclass, field

import numpy as np

from . import lib, shots
from .synth import Workload

# Largest step as a multiple of the 0.05 dm trial step (inversion.exe uses the
# same bound): the reference's parabola vertex is unbounded and can leave the
# physical range (inversion.cu:309-312).
STEP_BOUND = 8.0
# Trust region of the plain update: no cell's velocity changes by more than
# this fraction in one iteration.
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


def model_key(v) -> bytes:
    """Identity of a model's exact FP32 values."""
    return hashlib.blake2b(np.ascontiguousarray(v, np.float32).tobytes(), digest_size=16).digest()


def parabola_vertex(a, r):
    """Vertex of the parabola through (a_i, r_i), i = 0..2 (the reference's
    formula, inversion.cu:309-312); None when it is not a minimum."""
    num = (a[1] ** 2 - a[2] ** 2) * r[0] + (a[2] ** 2 - a[0] ** 2) * r[1] + (a[0] ** 2 - a[1] ** 2) * r[2]
    den = (a[1] - a[2]) * r[0] + (a[2] - a[0]) * r[1] + (a[0] - a[1]) * r[2]
    # positive second divided difference: a minimum
    convex = (r[2] - r[1]) / (a[2] - a[1]) > (r[1] - r[0]) / (a[1] - a[0])
    if den == 0 or not convex:
        return None
    return 0.5 * num / den


def search_step(misfit, trial, f0, a1, a2, cap):
    """Measured step search.  misfit(alpha) returns the misfit of trial step
    alpha; steps are capped at `cap`.  Returns (best step, its misfit), with
    (0, f0) when no candidate lowers the misfit."""
    a, f = [0.0], [f0]

    def measure(alpha):
        if alpha <= 0 or any(abs(alpha - x) <= 1e-12 * max(alpha, x) for x in a):
            return
        a.append(alpha)
        f.append(misfit(alpha))

    measure(min(a1, cap))
    measure(min(a2, cap))
    # expand while the misfit still falls at the largest step
    while len(a) > 2 and f[-1] < f[-2] and a[-1] < cap * (1 - 1e-12):
        measure(min(2.0 * a[-1], cap))
    # shrink when even the smallest trial is worse than no step
    for _ in range(2):
        if int(np.argmin(f)) != 0:
            break
        measure(0.25 * min(x for x in a if x > 0))
    order = np.argsort(a)
    a, f = [a[i] for i in order], [f[i] for i in order]
    k = int(np.argmin(f))
    if 0 < k < len(a) - 1:
        v = parabola_vertex(a[k - 1:k + 2], np.sqrt(f[k - 1:k + 2]))
        if v is not None and a[k - 1] < v < a[k + 1]:
            measure(min(v, cap))
    k = int(np.argmin(f))
    return (a[k], f[k]) if k else (0.0, f0)


class Fwi:
    """One inversion problem: geometry, observed data of this rank's shots,
    two library contexts (Cerjan boundary for the data, random boundary for
    the gradient).

    world/rank default to torch.distributed's when it is initialised.
    `contexts` replaces the two library contexts by objects with the same
    methods (the CPU tests of the cross-rank logic), with buffers on `device`."""

    def __init__(self, w: Workload, opts: FwiOptions | None = None, obs=None, world=None, rank=None,
                 contexts=None, device="cuda"):
        import torch
        self.torch = torch
        self.w, self.o = w, opts or FwiOptions()
        self.device = device
        if world is None:
            import torch.distributed as dist
            ok = dist.is_available() and dist.is_initialized()
            world, rank = (dist.get_world_size(), dist.get_rank()) if ok else (1, 0)
        self.world, self.rank = world, rank
        if contexts is None:
            flags = (lib.FLAG_GRAD_DY | lib.FLAG_SUBTRACT_SOURCE) if self.o.fixes else 0
            contexts = (lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_ABC,
                                    w.abc_factor, self.o.batch, 0),
                        lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC, 0.0,
                                    self.o.batch, flags))
        self.abc, self.rbc = contexts
        for c in (self.abc, self.rbc):
            c.set_geometry(w.src, w.rec, w.rec_first, w.rec_count)
        self.nshot = len(w.src)
        self.mine = shots.partition(self.nshot, world, rank)
        counts = [self.abc.shot_nrec(s) * w.nt for s in self.mine]
        self.offset = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        n = max(int(self.offset[-1]), 1)
        self.cal = torch.empty(n, device=device, dtype=torch.float32)
        self.res = torch.empty(n, device=device, dtype=torch.float32)      # residual of _res_key
        self.res_tmp = torch.empty(n, device=device, dtype=torch.float32)  # residual of _tmp_key
        self._res_key = self._tmp_key = None
        self._known = {}
        self.acc = None
        if world > 1:
            cells = self.rbc.nzz * self.rbc.nxx * self.rbc.nyy
            self.acc = (torch.empty(cells, device=device), torch.empty(cells, device=device))
        self.obs = obs if obs is not None else self.model(w.vp)
        self.evals = 0
        self.gradients = 0
        self.vbounds = (0.0, np.inf)

    # -- building blocks ------------------------------------------------------
    def _batches(self):
        """(position in self.mine, shot ids) of each launch."""
        B = self.o.batch
        return [(i, self.mine[i:i + B]) for i in range(0, len(self.mine), B)]

    def _ptr(self, buf, i):
        return buf.data_ptr() + 4 * int(self.offset[i])

    def model(self, v):
        """Seismograms of this rank's shots for velocity v (device tensor)."""
        out = self.torch.empty(max(int(self.offset[-1]), 1), device=self.device, dtype=self.torch.float32)
        self.abc.set_velocity(v)
        if self.device == "cuda":
            self.torch.cuda.synchronize()
        for i, b in self._batches():
            self.abc.model_shots_dev(b, self._ptr(out, i))
        return out

    def misfit(self, v) -> float:
        """sum (obs - cal)^2 over every shot of every rank (FP64).  The
        residual stays in res_tmp until adopt(v) keeps it."""
        self.abc.set_velocity(v)
        for i, b in self._batches():
            self.abc.model_shots_dev(b, self._ptr(self.cal, i))
        self.evals += 1
        local = self.abc.residual_dev(self.obs.data_ptr(), self.cal.data_ptr(), int(self.offset[-1]),
                                      self.res_tmp.data_ptr()) if len(self.mine) else 0.0
        f = shots.misfit_across_ranks(local)
        self._tmp_key = model_key(v)
        self._known[self._tmp_key] = f
        return f

    def adopt(self, v):
        """Keep the residual of v (the model just evaluated) for its gradient."""
        k = model_key(v)
        if self._tmp_key == k:
            self.res, self.res_tmp = self.res_tmp, self.res
            self._res_key, self._tmp_key = k, None

    def known_misfit(self, v) -> float:
        k = model_key(v)
        return self._known[k] if k in self._known else self.misfit(v)

    def gradient(self, v):
        """Misfit of v, then the gradient: returns (post-processed gradient,
        raw cropped gradient, cropped illumination, misfit)."""
        k = model_key(v)
        if self._res_key == k and k in self._known:
            f = self._known[k]
        else:
            f = self.misfit(v)
            self.adopt(v)
        self._known = {k: f}
        self.rbc.reset_accumulators()
        self.rbc.set_velocity(v)
        # shot s propagates through the pad of seed base + s: the pads depend
        # only on how many gradients came before, not on ranks or batches
        self.rbc.set_shot_random_boundary(base_seed=self.o.seed + 7919 * self.gradients, **self.o.rbc)
        for i, b in self._batches():
            self.rbc.gradient_shots_dev(b, self._ptr(self.res, i))
        if self.acc is not None:
            shots.reduce_context_accumulators(self.rbc, *self.acc)
        self.gradients += 1
        g, _ = self.rbc.gradient_post(self.o.zmask)
        raw, ill = self.rbc.get_accumulators()
        return g, crop(raw, self.w.nb), crop(ill, self.w.nb), f

    # -- plain line search ----------------------------------------------------
    def line_search(self, v, g, f0, dm):
        """Measured step on m = 1/v^2 along -g (search_step), within
        STEP_BOUND x 0.05 dm and the MAX_DV trust region.  Returns (new
        velocity, step, its measured misfit); the new model's residual is kept
        for its gradient."""
        if not (dm > 0) or not np.all(np.isfinite(g)) or not np.any(g):
            return v, 0.0, f0
        m = 1.0 / (v.astype(np.float64) ** 2)
        g64 = np.asarray(g, np.float64)
        lo, hi = self.vbounds
        def trial(alpha):
            # FP64 throughout, whatever the type of alpha: a Python float times
            # an FP32 array would round the product to FP32, so the same step
            # would give a slightly different model each way it is written
            return np.clip(1.0 / np.sqrt(np.maximum(m - float(alpha) * g64, 1e-12)), lo, hi).astype(np.float32)

        # largest step within the trust region, cell by cell in closed form:
        # v'/v = sqrt(m / (m - alpha g)) stays in [1 - MAX_DV, 1 + MAX_DV] for
        # alpha <= m (1 - 1/(1 + MAX_DV)^2) / g where g > 0 and
        # alpha <= m (1/(1 - MAX_DV)^2 - 1) / |g| where g < 0 (the clip to the
        # velocity bounds only shrinks a change)
        with np.errstate(divide="ignore"):
            lim = np.where(g64 > 0, m * (1.0 - 1.0 / (1.0 + MAX_DV) ** 2) / g64,
                           np.where(g64 < 0, m * (1.0 / (1.0 - MAX_DV) ** 2 - 1.0) / -g64, np.inf))
        cap = min(STEP_BOUND * 0.05 * dm, float(np.min(lim)))
        best = {}

        def f_of(alpha):
            vt = trial(alpha)
            f = self.misfit(vt)
            if f < best.get("f", f0):
                best["f"] = f
                self.adopt(vt)
            return f

        step, f = search_step(f_of, trial, f0, 0.02 * dm, 0.05 * dm, cap)
        if step == 0.0:
            return v, 0.0, f0
        return trial(step), float(step), f


def rms(v, ref) -> float:
    return float(np.sqrt(np.mean((v.astype(np.float64) - ref.astype(np.float64)) ** 2)))


def run(prob: Fwi, v0, iterations: int, learned=None, log=print):
    """Run `iterations` updates from v0.  With `learned` (a callable mapping
    (raw gradient, velocity, illumination) to a velocity update), each
    iteration also measures the misfit of v + learned(...) and keeps it only
    when it is at most the plain step's measured misfit.  Returns (final
    velocity, history)."""
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
                prob.adopt(v_l)
            hist[-1].update(f_learned=f_l)
        hist[-1].update(step=step, f_plain=f_plain, choice=choice, evals=prob.evals)
        log(f"iter {it}: misfit {f0:.6e} rms {hist[-1]['rms']:.2f} step {step:.3e} -> {choice}")
        v = v_next
    f = prob.known_misfit(v)
    hist.append(dict(iteration=iterations, misfit=f, rms=rms(v, w.vp), time=time.perf_counter() - t0,
                     evals=prob.evals))
    log(f"final: misfit {f:.6e} rms {hist[-1]['rms']:.2f} after {hist[-1]['time']:.1f} s")
    return v, hist
