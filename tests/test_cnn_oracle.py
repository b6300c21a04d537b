"""The CNN oracle itself (CPU): its analytic gradients against central finite
differences in FP64, so that it can pin the GPU gradients."""
import numpy as np

import cnn_oracle as co


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    nz, nx, ny = 6, 5, 4
    inp = rng.standard_normal((3, ny, nx, nz))
    tgt = rng.standard_normal((ny, nx, nz))
    W = np.zeros((4, 27, 16, 16))
    B = np.zeros((4, 16))
    for l in range(4):
        W[l, :, :co.COUT[l], :co.CIN[l]] = rng.standard_normal((27, co.COUT[l], co.CIN[l])) * 0.2
        B[l, :co.COUT[l]] = rng.standard_normal(co.COUT[l]) * 0.1
    _, gW, gB, _ = co.loss_and_grads(inp, tgt, W, B)
    e = 1e-5
    for (l, t, a, b) in [(0, 13, 2, 1), (1, 0, 5, 7), (2, 26, 15, 3), (3, 4, 0, 11), (3, 22, 0, 0)]:
        Wp, Wm = W.copy(), W.copy()
        Wp[l, t, a, b] += e
        Wm[l, t, a, b] -= e
        fd = (co.loss_and_grads(inp, tgt, Wp, B)[0] - co.loss_and_grads(inp, tgt, Wm, B)[0]) / (2 * e)
        assert abs(fd - gW[l, t, a, b]) <= 1e-6 * max(1.0, abs(fd))
    for l in range(4):
        Bp, Bm = B.copy(), B.copy()
        Bp[l, 0] += e
        Bm[l, 0] -= e
        fd = (co.loss_and_grads(inp, tgt, W, Bp)[0] - co.loss_and_grads(inp, tgt, W, Bm)[0]) / (2 * e)
        assert abs(fd - gB[l, 0]) <= 1e-6 * max(1.0, abs(fd))


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.0078125, 1.01171875, -3.3], np.float32)
    r = co.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[3] == 1.015625
    assert abs(r[4] + 3.3) < 0.02
