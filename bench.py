#!/usr/bin/env python
"""bench.py -- FD Mcell-updates/s and HBM roofline fraction on one B200 node.

Workload (default, the batched-RTM configuration): 201^3 model at 10 m, five
layers plus -8 %/+12 % Gaussian anomalies, smoothed migration model, 50-cell
random boundary (301^3 padded cells), nt = 2001 at 1 ms, Ricker 10 Hz peak
(N = 2120 time steps), 64 shots on an 8 x 8 grid with clipped 121 x 121
receiver patches.  One step = one batch of B shots (--batch, default 4) in
one launch per time step, each shot through its own new random boundary:
forward propagation, then the fused pass (source rebuilt backwards + adjoint
propagation + imaging), 3 x B padded cells x N steps of cell-updates.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B]
                  [--impl ours|reference] [--workload rtm|modeling]

Multi-GPU: one process per GPU (torchrun); shots are dealt round-robin to
ranks (weak scaling) and the images are summed with one NCCL all-reduce at
the end of the timed region; time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MEASURED = ROOT / "MEASURED_PEAKS.json"
TRAFFIC = ROOT / "profiles" / "traffic.json"
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    try:
        return float(json.loads(MEASURED.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                mx = float(p[1])
            except ValueError:
                continue
            for n, v in zip(names, p[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload(name, nt=None):
    """The benchmark workloads; nt shortens the time axis (profiling runs only)."""
    from fwi3d_b200 import synth
    kw = {} if nt is None else {"nt": nt}
    if name == "rtm":
        return synth.rtm_201(**kw)
    if name == "modeling":
        return synth.modeling_101(**kw)
    raise SystemExit(f"unknown workload {name}")


def cpu_baseline(w, n_steps=40):
    """FP64 oracle (OpenMP, all host cores) on a bounded sample of the same
    workload: n_steps forward + n_steps fused backward steps on the full padded
    grid.  Returns Mcell-updates/s."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    v = w.start if w.start is not None else w.vp
    vpp = orc.expand(v, w.nz, w.nx, w.ny, w.nb)
    nyy, nxx, nzz = vpp.shape
    wl, _ = orc.wavelet(n_steps, w.dt, w.fmax)
    src = orc.flat_index(nzz // 2, nxx // 2, nyy // 2, nzz, nxx)
    rec = np.array([src + 1], np.int64)
    t0 = time.perf_counter()
    _, P, Q = orc.forward(vpp, w.dh, w.dt, n_steps, 0, wl, src, rec)
    t1 = time.perf_counter()
    orc.backward(vpp, w.dh, w.dt, n_steps, 0, rec, np.zeros((1, n_steps)), P, Q)
    t2 = time.perf_counter()
    cells = nzz * nxx * nyy
    updates = cells * n_steps * 3
    return {"value": updates / (t2 - t0) / 1e6, "unit": "Mcell-updates/s", "cores": orc.num_threads(),
            "kind": "port",
            "sample": f"FP64 oracle, {n_steps} forward + {n_steps} fused backward steps on the "
                      f"{nzz}x{nxx}x{nyy} padded grid ({t2 - t0:.1f} s)"}


def run_ours(args, ws, rank, local):
    import torch
    from fwi3d_b200 import lib

    w = workload(args.workload, args.nt)
    rtm = args.workload == "rtm"
    B = args.batch if rtm else 1
    boundary = lib.BOUNDARY_RBC
    ctx = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, boundary, w.abc_factor, B, 0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.set_geometry(w.src, w.rec, w.rec_first, w.rec_count)
    ctx.set_velocity(w.start if w.start is not None else w.vp)
    # shot s propagates through the random pad of seed 1000 + s, rebuilt for
    # every batch inside the timed call (one velocity slot per batch slot)
    rbc = dict(w.rbc)
    ctx.set_shot_random_boundary(base_seed=1000, **rbc)
    if args.tiles:
        f, b = (int(x) for x in args.tiles.split(","))
        ctx.set_tiles(f, b)
    else:
        ctx.autotune()
    nsrc = len(w.src)
    N = ctx.tlag + w.nt
    cells = ctx.nzz * ctx.nxx * ctx.nyy
    updated = (ctx.nzz - 8) * (ctx.nxx - 8) * (ctx.nyy - 8)  # the 4-cell outer shell is never written
    updates_per_step = cells * N * (3 if rtm else 1) * B

    from fwi3d_b200 import shots as shotlib
    total = args.warmup + args.steps
    mine = shotlib.partition(nsrc, ws, rank)
    batches = [[mine[(k * B + j) % len(mine)] for j in range(B)] for k in range(total)]
    g = torch.Generator(device="cuda").manual_seed(1234 + rank)
    data = {}
    if rtm:
        for k, bt in enumerate(batches):
            key = tuple(bt)
            if key not in data:
                n = sum(ctx.shot_nrec(s) for s in bt) * w.nt
                data[key] = torch.randn(n, generator=g, device="cuda", dtype=torch.float32)
    seis_dev = None
    if not rtm:
        seis_dev = torch.empty(max(ctx.shot_nrec(s) for s in range(nsrc)) * w.nt, device="cuda")
    torch.cuda.synchronize()  # data come from the default stream; the library runs on `stream`

    def step(k, timing):
        bt = batches[k]
        if rtm:
            ctx.rtm_shots_dev(bt, data[tuple(bt)].data_ptr())
        else:
            ctx.model_shots_dev(bt, seis_dev.data_ptr())
        f, b = ctx.last_timing()
        timing[0] += f
        timing[1] += b

    tw = [0.0, 0.0]
    for k in range(args.warmup):
        step(k, tw)
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ctx.launch_count()
    timing = [0.0, 0.0]
    img_all = ill_all = None
    if ws > 1 and rtm:
        img_all = torch.empty(cells, device="cuda")
        ill_all = torch.empty(cells, device="cuda")
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            e0.record(stream)
            for k in range(args.warmup, total):
                step(k, timing)
            if img_all is not None:
                shotlib.reduce_context_accumulators(ctx, img_all, ill_all)
            e1.record(stream)
        torch.cuda.synchronize()
    launches = ctx.launch_count() - launches0
    barrier(ws)
    ms_local = e0.elapsed_time(e1)
    ms = max_over_ranks(ms_local, ws)
    value = updates_per_step * args.steps * ws / (ms / 1e3) / 1e6

    # roofline of the dominant kernel: the fused backward step for RTM (28 B
    # per cell-step for the four wavefield levels and the stencil coefficient,
    # plus 16 B for the image and illumination of every cell of the physical
    # box, the only cells that accumulate), the forward step (16 B per
    # cell-update) for modeling
    peak, peak_kind = hbm_peak()
    # per launch: B shots of the padded grid; frac_updated charges the field
    # bytes only to the cells a launch writes (the outer 4-cell shell is read,
    # never written)
    box = w.nz * w.nx * w.ny
    if rtm:
        kern_ms = timing[1] / args.steps / N
        bytes_per_launch = (28.0 * cells + 16.0 * box) * B
        bytes_updated = (28.0 * updated + 16.0 * box) * B
        name = "fd_backward_kernel"
    else:
        kern_ms = timing[0] / args.steps / N
        bytes_per_launch = 16.0 * cells * B
        bytes_updated = 16.0 * updated * B
        name = "fd_forward_kernel"
    achieved = bytes_per_launch / (kern_ms / 1e3) / 1e9
    achieved_upd = bytes_updated / (kern_ms / 1e3) / 1e9
    traffic = None
    try:
        tr = json.loads(TRAFFIC.read_text())
        if name in tr:
            traffic = float(tr[name]["bytes_per_cell"]) * cells * B
    except Exception:
        pass
    fwd_ms = timing[0] / args.steps / N
    fwd_upd = 16.0 * updated * B / (fwd_ms / 1e3) / 1e9
    roof = {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
            "achieved_updated": round(achieved_upd, 1), "frac_updated": round(achieved_upd / peak, 4),
            "traffic": traffic, "algorithmic_bytes": bytes_per_launch,
            "algorithmic_bytes_updated": bytes_updated, "accumulated_cells_per_shot": box if rtm else 0,
            "launch_ms": round(kern_ms, 5), "shots_per_launch": B,
            "forward_kernel": {"achieved": round(16.0 * cells * B / (fwd_ms / 1e3) / 1e9, 1),
                               "frac": round(16.0 * cells * B / (fwd_ms / 1e3) / 1e9 / peak, 4),
                               "achieved_updated": round(fwd_upd, 1), "frac_updated": round(fwd_upd / peak, 4),
                               "launch_ms": round(fwd_ms, 5)}}

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        host = {}
        for bt in batches[args.warmup:]:
            key = tuple(bt)
            if key in host:
                continue
            n = sum(ctx.shot_nrec(s) for s in bt) * w.nt
            pin = torch.empty(n, dtype=torch.float32, pin_memory=True)
            if rtm:
                pin.copy_(data[key].cpu())
            host[key] = pin
        out = torch.empty(w.nz * w.nx * w.ny if rtm else max(ctx.shot_nrec(s) for s in range(nsrc)) * w.nt,
                          dtype=torch.float32, pin_memory=True)
        h2d = d2h = 0
        dev_ms = 0.0  # the propagation kernels' share of it (their CUDA events)
        barrier(ws)
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            e0.record(stream)
            for k in range(args.warmup, total):
                bt = batches[k]
                if rtm:
                    ctx.rtm_shots(bt, host[tuple(bt)].numpy())
                    dev_ms += sum(ctx.last_timing())
                    ctx.rtm_image(out=out.numpy())  # straight into the pinned host buffer
                    h2d += host[tuple(bt)].numel() * 4
                    d2h += out.numel() * 4
                else:
                    r = ctx.model_shots(bt)[0]
                    d2h += r.size * 4
            e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), ws)
        wall = time.perf_counter() - t0
        e2e = {"value": round(updates_per_step * args.steps * ws / (e2e_ms / 1e3) / 1e6, 1),
               "unit": "Mcell-updates/s", "h2d_bytes_per_step": h2d // args.steps,
               "d2h_bytes_per_step": d2h // args.steps, "wall_s": round(wall, 3),
               "propagation_ms_per_step": round(dev_ms / args.steps, 3) if rtm else None}

    if rank != 0:
        return None
    field_mb = ctx.nzz * ctx.nxx * ctx.nyy * 4 / 1e6
    nfields = 7 if rtm else 3  # forward: two time levels + velocity; RTM adds two adjoint levels + two accumulators
    ws_mb = field_mb * nfields
    l2_note = (f"working set {nfields} fields x {field_mb:.0f} MB = {ws_mb:.0f} MB per shot, "
               + ("larger than the 126 MB L2" if ws_mb > 126 else
                  "below the 126 MB L2: fields stay partly L2-resident between time steps"))
    line = {
        "metric": "FD Mcell-updates/s", "value": round(value, 1), "unit": "Mcell-updates/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded layered model with Gaussian anomalies, seeded random observed data",
        "config": {
            "workload": (f"{w.name}: padded {ctx.nzz}x{ctx.nxx}x{ctx.nyy}, nt={w.nt}, N={N} steps; "
                         + (f"one batch of {B} shots per step, in one launch per time step, each shot through its "
                            "own new random boundary: forward + fused backward (3 cell-updates per padded cell, "
                            "time step and shot)" if rtm else "one shot per step: forward modeling")),
            "shots": nsrc, "shots_per_step": B, "shots_per_launch": B, "l2": l2_note,
            "tiles": ctx.tiles(), "parallelism": f"shots/{ws}"},
        "roofline": roof,
        "e2e": e2e,
        "gpu_launches": int(launches),
    }
    return line, clocks.summary()


def secondary_modeling(steps=5, warmup=2):
    """The plain-modeling configuration (101^3 model + 50-cell random pad,
    201^3 padded cells, nt = 1001, N = 1120, one shot, 51 x 51 receivers),
    measured in the same run: device time per shot with CUDA events on the
    library's stream, and the forward kernel's HBM fraction.  Its working set
    (3 fields x 32.5 MB) fits in the 126 MB L2."""
    import torch
    from fwi3d_b200 import lib
    w = workload("modeling")
    ctx = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC, w.abc_factor, 1, 0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.set_geometry(w.src, w.rec)
    ctx.set_velocity(w.vp)
    ctx.set_shot_random_boundary(base_seed=1, **w.rbc)
    ctx.autotune()
    seis = torch.empty(len(w.rec) * w.nt, device="cuda")
    torch.cuda.synchronize()
    for _ in range(warmup):
        ctx.model_shots_dev([0], seis.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fwd = 0.0
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(steps):
            ctx.model_shots_dev([0], seis.data_ptr())
            fwd += ctx.last_timing()[0]
        e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    N = ctx.tlag + w.nt
    cells = ctx.nzz * ctx.nxx * ctx.nyy
    updated = (ctx.nzz - 8) * (ctx.nxx - 8) * (ctx.nyy - 8)
    peak, _ = hbm_peak()
    kern = fwd / steps / N
    ctx.close()
    return {"workload": f"{w.name}: padded {cells ** (1 / 3):.0f}^3, nt={w.nt}, N={N}, one shot, "
                        f"{len(w.rec)} receivers; random pad",
            "value": round(cells * N / (ms / 1e3) / 1e6, 1), "unit": "Mcell-updates/s",
            "ms_per_step": round(ms, 3), "steps": steps, "warmup": warmup,
            "forward_kernel": {"launch_ms": round(kern, 5),
                               "frac": round(16.0 * cells / (kern / 1e3) / 1e9 / peak, 4),
                               "frac_updated": round(16.0 * updated / (kern / 1e3) / 1e9 / peak, 4)},
            "l2": "working set 3 fields x 32.5 MB, below the 126 MB L2"}


def run_reference(args, ws, rank, local):
    """The reference's own CUDA build (oracle/_ref, compiled from its sources)
    on the same workload: per step, Modeling::forward_solver plus the
    Migration::backward_propagation loop of inject_seismogram +
    cross_correlation, timed with CUDA events around the two time loops."""
    if rank != 0:
        return None
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    if not orc.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_fwi3d.so was not built "
                "(reference sources absent when building)"}, None
    w = workload(args.workload)
    rtm = args.workload == "rtm"
    v = w.start if w.start is not None else w.vp
    vpp = orc.expand(v, w.nz, w.nx, w.ny, w.nb).astype(np.float32)
    nyy, nxx, nzz = vpp.shape
    # the same kind of pad as ours, generated host-side (ramped +-30 %)
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    nb = w.nb

    def ramp(n):
        i = np.arange(n)
        d = np.where(i < nb, nb - i, np.where(i >= n - nb, i - (n - nb - 1), 0))
        return d / nb

    r = np.maximum(np.maximum(ramp(nyy)[:, None, None], ramp(nxx)[None, :, None]), ramp(nzz)[None, None, :])
    vpp = (vpp * (1 + 0.3 * r * np.random.default_rng(5).uniform(-1, 1, vpp.shape))).astype(np.float32)
    lim = 0.98 * 2 / np.sqrt(3 * 6.501) * w.dh / w.dt
    vpp = np.minimum(vpp, lim).astype(np.float32)
    nsrc = len(w.src)
    total = args.warmup + args.steps
    shots = [k % nsrc for k in range(total)]
    tmp = tempfile.mkdtemp()
    cells = nzz * nxx * nyy
    ms_sum = 0.0
    N = None
    with ClockSampler(local) as clocks:
        for k, s in enumerate(shots):
            f, c = (w.rec_first[s], w.rec_count[s]) if w.rec_first is not None else (0, len(w.rec))
            rec = w.rec[f:f + c]
            params = orc.write_reference_setup(Path(tmp) / f"s{k}", w.nz, w.nx, w.ny, w.dh, w.nt, w.dt, w.fmax,
                                               w.nb, w.src[s:s + 1], rec)
            adj = np.random.default_rng(s).standard_normal((len(rec), w.nt)).astype(np.float32) if rtm else None
            out = orc.ref_run(params, vpp, shot=0, abc=not rtm, backward=1 if rtm else 0, adj=adj)
            N = out["tlag"] + w.nt
            if k >= args.warmup:
                ms_sum += float(out["ms"][0] + out["ms"][1])
    updates = cells * N * (3 if rtm else 1) * args.steps
    value = updates / (ms_sum / 1e3) / 1e6
    line = {"impl": "reference", "metric": "FD Mcell-updates/s", "value": round(value, 1),
            "unit": "Mcell-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_sum / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 storage, f64 stencil arithmetic", "data": "synthetic",
            "config": {"workload": f"{w.name}: padded {nzz}x{nxx}x{nyy}, nt={w.nt}, N={N}; reference CUDA "
                                   "build (sm_100a) of FWI3D's own kernels, device time of its time loops"},
            "cpu_baseline": {"value": round(value, 1), "unit": "Mcell-updates/s", "cores": 0,
                             "kind": "reference",
                             "sample": "reference CUDA build on the GPU (the reference has no CPU path)"},
            "e2e": {"value": round(value, 1), "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    return line, clocks.summary()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["rtm", "modeling"], default="rtm")
    ap.add_argument("--batch", type=int, default=4, help="shots per launch (RTM)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the plain-modeling (101^3 + 50-cell pad) secondary measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    ap.add_argument("--tiles", default="", help="fixed forward,backward tile indices instead of autotuning")
    ap.add_argument("--nt", type=int, default=None, help="shorter time axis for profiling runs (not a bench number)")
    args = ap.parse_args()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        res = run_reference(args, ws, rank, local)
    else:
        res = run_ours(args, ws, rank, local)
    if rank == 0 and res is not None:
        line, clocks = res
        if clocks is not None:
            line["clocks"] = clocks
        if args.impl == "ours" and ws == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(workload(args.workload))
        if args.impl == "ours" and ws == 1 and args.workload == "rtm" and not args.no_secondary:
            line["secondary"] = secondary_modeling()
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
