"""The learned preconditioner network (fwi_cnn_*) against its FP64 oracle
(oracle/cnn_oracle.py): forward values, weight and bias gradients, and
training progress.  BF16 tolerances are stated per check."""
import numpy as np
import pytest

import cnn_oracle as co
from cases import rel_l2
from fwi3d_b200 import lib

pytestmark = pytest.mark.gpu

SHAPE = (20, 12, 10)  # nz, nx, ny: one full and one partial 16-voxel z tile


def _inputs(seed=0, shape=SHAPE):
    nz, nx, ny = shape
    rng = np.random.default_rng(seed)
    inp = rng.standard_normal((3, ny, nx, nz)).astype(np.float32)
    target = (0.3 * inp[0] - 0.2 * np.roll(inp[1], 1, axis=2) + 0.1).astype(np.float32)
    return inp, target


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _random_weights(net, seed):
    rng = np.random.default_rng(seed)
    w, b = net.get_weights()
    w = (w != 0) * rng.standard_normal(w.shape).astype(np.float32) * 0.15
    b = rng.standard_normal(b.shape).astype(np.float32) * 0.05
    net.set_weights(w, b)
    return net.get_weights()


def test_forward_matches_oracle():
    import torch
    net = lib.Cnn(seed=1)
    w, b = _random_weights(net, 2)
    inp, _ = _inputs(3)
    x = _dev(inp)
    out = torch.empty(inp[0].size, device="cuda")
    net.forward(SHAPE, x.data_ptr(), out.data_ptr())
    got = out.cpu().numpy().reshape(inp.shape[1:])
    ref_bf, _ = co.forward(inp, w, b, round_bf16=True)
    ref64, _ = co.forward(inp, w, b, round_bf16=False)
    # same BF16 rounding points as the GPU: only FP32-vs-FP64 accumulation differs
    assert rel_l2(got, ref_bf) < 2e-3
    # against exact FP64 arithmetic: the BF16 storage error
    assert rel_l2(got, ref64) < 3e-2


def test_gradients_match_oracle():
    net = lib.Cnn(seed=4)
    w, b = _random_weights(net, 5)
    inp, target = _inputs(6)
    x, t = _dev(inp), _dev(target)
    loss, gw, gb = net.train_step(SHAPE, x.data_ptr(), t.data_ptr(), 0.0, want_grads=True)
    rloss, rgw, rgb, _ = co.loss_and_grads(inp, target, w, b, round_bf16=True)
    assert abs(loss - rloss) <= 2e-3 * rloss
    for l in range(4):
        assert rel_l2(gw[l], rgw[l]) < 1e-2, (l, rel_l2(gw[l], rgw[l]))
        assert rel_l2(gb[l][: co.COUT[l]], rgb[l][: co.COUT[l]]) < 1e-2
    _, fgw, _, _ = co.loss_and_grads(inp, target, w, b, round_bf16=False)
    for l in range(4):
        assert rel_l2(gw[l], fgw[l]) < 6e-2


def test_padding_channels_stay_zero_and_training_lowers_the_loss():
    net = lib.Cnn(seed=7)
    inp, target = _inputs(8, (32, 16, 16))
    x, t = _dev(inp), _dev(target)
    losses = [net.train_step((32, 16, 16), x.data_ptr(), t.data_ptr(), 3e-3) for _ in range(60)]
    assert losses[-1] < 0.5 * losses[0], losses[::10]
    w, b = net.get_weights()
    assert np.all(w[0][:, :, 3:] == 0) and np.all(w[3][:, 1:, :] == 0) and np.all(b[3][1:] == 0)


def test_training_step_is_reproducible():
    """Fixed-order partial sums: the same step twice gives the same bits."""
    net = lib.Cnn(seed=9)
    inp, target = _inputs(10)
    x, t = _dev(inp), _dev(target)
    a = net.train_step(SHAPE, x.data_ptr(), t.data_ptr(), 0.0, want_grads=True)
    b = net.train_step(SHAPE, x.data_ptr(), t.data_ptr(), 0.0, want_grads=True)
    assert a[0] == b[0]
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


def test_forward_matches_oracle_when_tile_runs_cross_planes():
    """A volume whose y planes hold many 120-row tile positions, so that the
    persistent CTAs' tile ranges start and end inside planes."""
    import torch
    shape = (40, 36, 30)
    net = lib.Cnn(seed=11)
    w, b = _random_weights(net, 12)
    inp, _ = _inputs(13, shape)
    x = _dev(inp)
    out = torch.empty(inp[0].size, device="cuda")
    net.forward(shape, x.data_ptr(), out.data_ptr())
    got = out.cpu().numpy().reshape(inp.shape[1:])
    ref_bf, _ = co.forward(inp, w, b, round_bf16=True)
    assert rel_l2(got, ref_bf) < 2e-3
