"""FP64 numpy oracle of the learned preconditioner network -- TEST
INFRASTRUCTURE ONLY (checks fwi_cnn_* in libfwi3d.so; never used by it).

Network: 4 conv3d layers, 3 -> 16 -> 16 -> 16 -> 1 channels, 3^3 taps with
zero "same" padding, ReLU after the first three, loss 0.5 mean (f - target)^2.
Arrays: volumes (ny, nx, nz[, C]) C-order (z fastest); weights
[4][27][16 co][16 ci] with tap t = (dz+1) + 3(dx+1) + 9(dy+1); biases [4][16].

With bf16=True the oracle rounds to bfloat16 (round to nearest even) at the
points where the GPU stores BF16: the packed input, the weights, every hidden
activation, the loss gradient and every propagated data gradient; all sums
stay FP64.
"""
from __future__ import annotations

import numpy as np

CIN = [3, 16, 16, 16]
COUT = [16, 16, 16, 1]
TAPS = [(dz, dx, dy) for dy in (-1, 0, 1) for dx in (-1, 0, 1) for dz in (-1, 0, 1)]


def bf16(a):
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def shift(x, dz, dx, dy):
    """s[k, j, i] = x[k + dy, j + dx, i + dz], zero outside."""
    out = np.zeros_like(x)
    ny, nx, nz = x.shape[:3]

    def sl(d, n):
        return (slice(max(0, -d), n - max(0, d)), slice(max(0, d), n - max(0, -d)))

    (ok, ik), (oj, ij), (oi, ii) = sl(dy, ny), sl(dx, nx), sl(dz, nz)
    out[ok, oj, oi] = x[ik, ij, ii]
    return out


def conv(x, W, b=None, sign=1):
    """y[v, co] = sum_t sum_ci x[v + sign*off_t, ci] W[t, co, ci] (+ b)."""
    y = np.zeros(x.shape[:3] + (W.shape[1],))
    for t, (dz, dx, dy) in enumerate(TAPS):
        y += shift(x, sign * dz, sign * dx, sign * dy) @ W[t].T
    return y if b is None else y + b


def pack(inp):
    """(3, ny, nx, nz) channels -> (ny, nx, nz, 16)."""
    x = np.zeros(inp.shape[1:] + (16,))
    x[..., :3] = np.moveaxis(inp, 0, -1)
    return x


def forward(inp, W, B, round_bf16=False):
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
    acts = [r(pack(inp))]
    for l in range(4):
        z = conv(acts[-1], r(W[l]), B[l])
        if l < 3:
            acts.append(r(np.maximum(z, 0.0)))
        else:
            pred = z[..., 0]
    return pred, acts


def loss_and_grads(inp, target, W, B, round_bf16=False):
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
    pred, acts = forward(inp, W, B, round_bf16)
    V = pred.size
    d = pred - target
    loss = 0.5 * np.sum(d * d) / V
    dy = np.zeros(pred.shape + (16,))
    dy[..., 0] = r(d)
    gW = np.zeros((4, 27, 16, 16))
    gB = np.zeros((4, 16))
    for l in range(3, -1, -1):
        x = acts[l]
        for t, (dz, dx, dy_) in enumerate(TAPS):
            xs = shift(x, dz, dx, dy_)
            gW[l, t] = np.einsum("kjic,kjid->cd", dy, xs) / V
        gB[l] = dy.reshape(-1, 16).sum(0) / V
        if l > 0:
            Wt = np.transpose(r(W[l]), (0, 2, 1))  # [t][ci][co]
            dx_ = conv(dy, Wt, sign=-1)
            dy = r(dx_ * (acts[l] > 0))
    for l in range(4):
        gW[l, :, COUT[l]:, :] = 0.0
        gW[l, :, :, CIN[l]:] = 0.0
        gB[l, COUT[l]:] = 0.0
    return loss, gW, gB, pred
