"""Learned gradient preconditioner: data, training and use inside FWI.

Pairs come from the project's own FWI on seeded random models (synth.cnn_128):
inputs are the raw gradient, the velocity and the illumination at a model v,
the target is true - v.  Each model gives pairs at the smoothed start model
and at a partly corrected model v = start + s (true - start), s drawn from
[0.3, 0.8), so that at a later iterate the network predicts the remaining
correction instead of the whole one again.  The network is fwi_cnn_* in
libfwi3d.so (BF16 tensor cores, FP32 accumulation, FP32 Adam).

    python -m fwi3d_b200.precond pipeline --models 0:200 --weights W.npz --report R.json
    python -m fwi3d_b200.precond compare --weights W.npz --iterations 5 --out C.json
    python -m fwi3d_b200.precond time --n 128 --steps 20 --warmup 2

Input normalisation (per volume): the raw gradient below the depth mask,
divided by its 99.5th percentile of |g| and clipped to [-4, 4]; (v - 2500)/1000;
log10(illum / max illum + 1e-6)/3 + 1.  Output scale: 200 m/s.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

from . import fwi, lib, synth

DV_SCALE = 200.0


def features(raw, v, ill, zmask_cells=0):
    g = raw.copy()
    g[:, :, : zmask_cells + 1] = 0.0
    scale = float(np.percentile(np.abs(g), 99.5))
    g = np.clip(g / max(scale, 1e-30), -4.0, 4.0)
    vv = (v - 2500.0) / 1000.0
    il = np.log10(ill / max(float(ill.max()), 1e-30) + 1e-6) / 3.0 + 1.0
    return np.stack([g, vv, il]).astype(np.float32)


def pair_from(w: synth.Workload, batch: int, seed: int, s: float = 0.0, prob=None):
    """(features, target, misfit) at v = start + s (true - start)."""
    prob = prob or fwi.Fwi(w, fwi.FwiOptions(batch=batch, seed=seed, zmask=w.zmask, rbc=w.rbc))
    v = (w.start.astype(np.float64) + s * (w.vp.astype(np.float64) - w.start)).astype(np.float32)
    _, raw, ill, f = prob.gradient(v)
    x = features(raw, v, ill, int(w.zmask / w.dh))
    y = ((w.vp - v) / DV_SCALE).astype(np.float32)
    return x, y, f


def stages(index: int) -> list[float]:
    """The models a training model contributes pairs at: the start model and
    one partly corrected model (seeded by the model index)."""
    return [0.0, float(np.random.default_rng(7000 + index).uniform(0.3, 0.8))]


def training_pairs(index: int, nt: int = 1201, batch: int = 9):
    """Pairs of training model `index` (one FWI problem, its observed data
    modelled once)."""
    w = synth.cnn_128(index, nt=nt)
    prob = fwi.Fwi(w, fwi.FwiOptions(batch=batch, seed=index, zmask=w.zmask, rbc=w.rbc))
    return [pair_from(w, batch, index, s, prob) for s in stages(index)]


class Learned:
    """Callable (raw gradient, velocity, illumination) -> velocity update."""

    def __init__(self, net: lib.Cnn, zmask_cells=0):
        import torch
        self.net, self.torch, self.zc = net, torch, zmask_cells

    def __call__(self, raw, v, ill):
        x = self.torch.from_numpy(features(raw, v, ill, self.zc)).cuda()
        out = self.torch.empty(v.size, device="cuda")
        ny, nx, nz = v.shape
        self.net.forward((nz, nx, ny), x.data_ptr(), out.data_ptr())
        return (out.cpu().numpy().reshape(v.shape) * DV_SCALE).astype(np.float32)


def save_weights(net: lib.Cnn, path):
    w, b = net.get_weights()
    np.savez_compressed(path, w=w, b=b)


def load_weights(path, seed=0) -> lib.Cnn:
    d = np.load(path)
    net = lib.Cnn(seed)
    net.set_weights(d["w"], d["b"])
    return net


def train(xs, ys, epochs=40, lr=2e-3, seed=0, log=print):
    """Adam over the pairs, one volume per step, cosine-decayed learning rate."""
    import torch
    net = lib.Cnn(seed)
    rng = np.random.default_rng(seed)
    dev = [(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()) for x, y in zip(xs, ys)]
    ny, nx, nz = xs[0].shape[1:]
    steps = epochs * len(dev)
    k = 0
    hist = []
    for ep in range(epochs):
        tot = 0.0
        for i in rng.permutation(len(dev)):
            cur = lr * 0.5 * (1 + np.cos(np.pi * k / steps))
            tot += net.train_step((nz, nx, ny), dev[i][0].data_ptr(), dev[i][1].data_ptr(), cur)
            k += 1
        hist.append(tot / len(dev))
        if ep % 10 == 0 or ep == epochs - 1:
            log(f"epoch {ep}: loss {hist[-1]:.5f}")
    return net, hist


def evaluate(net, xs, ys):
    """Mean relative L2 error of the predicted update (1.0 = predicting zero)."""
    import torch
    errs = []
    for x, y in zip(xs, ys):
        xd = torch.from_numpy(x).cuda()
        out = torch.empty(y.size, device="cuda")
        ny, nx, nz = y.shape
        net.forward((nz, nx, ny), xd.data_ptr(), out.data_ptr())
        p = out.cpu().numpy().reshape(y.shape)
        errs.append(float(np.linalg.norm(p - y) / np.linalg.norm(y)))
    return float(np.mean(errs))


def summarise(plain, learned):
    """Wall time for the learned run to reach the plain run's final misfit,
    with the model RMS error of both at that point; and the same at the plain
    run's final model RMS error."""
    target = plain[-1]["misfit"]
    hit = next((h for h in learned if h["misfit"] <= target), None)
    out = {"plain_final_misfit": target, "plain_final_rms": plain[-1]["rms"], "plain_time": plain[-1]["time"],
           "start_rms": plain[0]["rms"],
           "learned_final_misfit": learned[-1]["misfit"], "learned_final_rms": learned[-1]["rms"],
           "learned_time": learned[-1]["time"], "learned_max_rms": max(h["rms"] for h in learned),
           "learned_choices": [h.get("choice") for h in learned[:-1]]}
    if hit is not None:
        out.update(learned_time_to_plain_misfit=hit["time"], learned_rms_at_that_point=hit["rms"],
                   time_ratio=hit["time"] / plain[-1]["time"])
    hit_rms = next((h for h in learned if h["rms"] <= plain[-1]["rms"]), None)
    if hit_rms is not None:
        out.update(learned_time_to_plain_rms=hit_rms["time"], time_ratio_at_equal_rms=hit_rms["time"] / plain[-1]["time"])
    return out


def time_network(n=128, steps=20, warmup=2, seed=0):
    """Device time of the network on an n^3 volume (CUDA events): forward
    (input packing + 4 layers) and a training step (forward, loss, backward,
    Adam).  Random inputs; each warm-up step is one forward + one training
    step at lr 0."""
    import torch
    net = lib.Cnn(seed)
    shape = (n, n, n)
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn(3, n, n, n, device="cuda", generator=g)
    y = torch.randn(n, n, n, device="cuda", generator=g) * 0.1
    out = torch.empty(n, n, n, device="cuda")
    for _ in range(warmup):
        net.forward(shape, x.data_ptr(), out.data_ptr())
        net.train_step(shape, x.data_ptr(), y.data_ptr(), 0.0)
    torch.cuda.synchronize()

    def timed(f):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            f()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    fwd = timed(lambda: net.forward(shape, x.data_ptr(), out.data_ptr()))
    trn = timed(lambda: net.train_step(shape, x.data_ptr(), y.data_ptr(), 1e-5))
    flop = 2 * 27 * (3 * 16 + 16 * 16 + 16 * 16 + 16 * 1) * n ** 3
    return {"n": n, "steps": steps, "forward_ms": fwd, "train_step_ms": trn,
            "forward_tflops_algorithmic": flop / (fwd * 1e-3) / 1e12}


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    pl = sub.add_parser("pipeline", help="generate pairs in memory, train, save weights and a report")
    pl.add_argument("--models", default="0:200")
    pl.add_argument("--nt", type=int, default=1201)
    pl.add_argument("--holdout", type=int, default=8)
    pl.add_argument("--epochs", type=int, default=150)
    pl.add_argument("--lr", type=float, default=3e-3)
    pl.add_argument("--fwi-holdout", type=int, default=2, help="held-out models also run through FWI")
    pl.add_argument("--weights", required=True)
    pl.add_argument("--report", required=True)
    c = sub.add_parser("compare")
    c.add_argument("--weights", required=True)
    c.add_argument("--iterations", type=int, default=5)
    c.add_argument("--workload", default="fwi_301")
    c.add_argument("--nt", type=int, default=2001)
    c.add_argument("--batch", type=int, default=4)
    c.add_argument("--out", required=True)
    t = sub.add_parser("time", help="device time of the network's forward and training step")
    t.add_argument("--n", type=int, default=128)
    t.add_argument("--steps", type=int, default=20)
    t.add_argument("--warmup", type=int, default=2)
    a = ap.parse_args(argv)

    if a.cmd == "pipeline":
        lo, hi = (int(x) for x in a.models.split(":"))
        t0 = time.perf_counter()
        xs, ys = [], []
        for i in range(lo, hi):
            for x, y, f in training_pairs(i, a.nt):
                xs.append(x)
                ys.append(y)
            if i % 16 == 0:
                print(f"model {i}: misfit {f:.4e} ({time.perf_counter() - t0:.1f} s)", flush=True)
        t_data = time.perf_counter() - t0
        # hold out whole models (both of their pairs)
        h = a.holdout * len(stages(lo))
        t1 = time.perf_counter()
        net, hist = train(xs[h:], ys[h:], epochs=a.epochs, lr=a.lr)
        t_train = time.perf_counter() - t1
        save_weights(net, a.weights)
        res = {"models": [lo, hi], "nt": a.nt, "train_pairs": len(xs) - h, "holdout_pairs": h,
               "stages": "start model and start + s (true - start), s in [0.3, 0.8)",
               "epochs": a.epochs, "data_seconds": t_data, "train_seconds": t_train,
               "loss_first_last": [hist[0], hist[-1]], "loss_history": hist,
               "holdout_rel_error": evaluate(net, xs[:h], ys[:h]),
               "train_rel_error": evaluate(net, xs[h:h + 8], ys[h:h + 8]), "fwi_holdout": []}
        del xs, ys
        for i in range(lo, lo + a.fwi_holdout):
            w = synth.cnn_128(i, nt=a.nt)
            prob = fwi.Fwi(w, fwi.FwiOptions(batch=9, seed=500 + i, zmask=w.zmask, rbc=w.rbc))
            _, hp = fwi.run(prob, w.start, 3)
            _, hl = fwi.run(prob, w.start, 3, learned=Learned(net, int(w.zmask / w.dh)))
            res["fwi_holdout"].append({"model": i, **summarise(hp, hl), "plain": hp, "learned": hl})
        Path(a.report).write_text(json.dumps(res, indent=1))
        print(json.dumps({k: v for k, v in res.items() if k not in ("loss_history", "fwi_holdout")}), flush=True)
        for r in res["fwi_holdout"]:
            print(json.dumps({k: v for k, v in r.items() if k not in ("plain", "learned")}), flush=True)
    elif a.cmd == "time":
        print(json.dumps(time_network(a.n, a.steps, a.warmup)), flush=True)
    elif a.cmd == "compare":
        w = getattr(synth, a.workload)(nt=a.nt)
        prob = fwi.Fwi(w, fwi.FwiOptions(batch=a.batch, zmask=w.zmask, rbc=w.rbc))
        net = load_weights(a.weights)
        out = {"workload": w.name, "iterations": a.iterations}
        _, out["plain"] = fwi.run(prob, w.start, a.iterations)
        _, out["learned"] = fwi.run(prob, w.start, a.iterations, learned=Learned(net, int(w.zmask / w.dh)))
        out["summary"] = summarise(out["plain"], out["learned"])
        Path(a.out).write_text(json.dumps(out, indent=1))
        print(json.dumps(out["summary"]), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
