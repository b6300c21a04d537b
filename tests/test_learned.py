"""What the learned preconditioner gains over the plain method.

The network is trained on the GPU, by the project's own kernels, on pairs
that the project's own FWI produces on seeded random 48^3 models (raw
gradient, velocity, illumination at the start model and at a partly
corrected model -> true - current velocity).  On held-out models, FWI with
the learned step (kept only when its measured misfit is at most the plain
step's measured misfit) must lower the misfit clearly more on average, never
end above the plain method's misfit, and not end with a larger model error."""
import numpy as np
import pytest

from fwi3d_b200 import fwi, precond, synth

pytestmark = pytest.mark.gpu

HOLDOUT = 6
TRAIN = 30


@pytest.fixture(scope="module")
def trained():
    xs, ys = [], []
    for i in range(HOLDOUT, HOLDOUT + TRAIN):
        w = synth.small_fwi(i)
        prob = fwi.Fwi(w, fwi.FwiOptions(batch=4, seed=i, rbc=w.rbc, zmask=w.zmask))
        for s in precond.stages(i):
            x, y, _ = precond.pair_from(w, 4, i, s, prob)
            xs.append(x)
            ys.append(y)
    net, hist = precond.train(xs, ys, epochs=80, lr=3e-3, log=lambda *a: None)
    assert hist[-1] < 0.5 * hist[0]
    return net


def test_learned_step_beats_plain_fwi_on_held_out_models(trained):
    ratios, rms_ratios = [], []
    for i in range(HOLDOUT):
        w = synth.small_fwi(i)
        prob = fwi.Fwi(w, fwi.FwiOptions(batch=4, seed=100 + i, rbc=w.rbc, zmask=w.zmask))
        _, hp = fwi.run(prob, w.start, 2, log=lambda *a: None)
        _, hl = fwi.run(prob, w.start, 2, learned=precond.Learned(trained, int(w.zmask / w.dh)),
                        log=lambda *a: None)
        assert hp[0]["misfit"] == hl[0]["misfit"]
        for h, nxt in zip(hl[:-1], hl[1:]):
            # the accept rule: the plain step's measured misfit, no slack
            assert (h["choice"] == "learned") == (h["f_learned"] <= h["f_plain"])
            assert nxt["misfit"] == min(h["f_learned"], h["f_plain"])
        ratios.append(hl[-1]["misfit"] / hp[-1]["misfit"])
        rms_ratios.append(hl[-1]["rms"] / hp[-1]["rms"])
    ratios, rms_ratios = np.array(ratios), np.array(rms_ratios)
    print("learned / plain misfit after 2 iterations:", np.round(ratios, 3))
    print("learned / plain model RMS error after 2 iterations:", np.round(rms_ratios, 3))
    assert ratios.max() <= 1.0, ratios
    assert ratios.mean() < 0.8, ratios
    assert rms_ratios.mean() <= 1.0, rms_ratios
