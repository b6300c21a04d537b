"""FWI driver logic on CPU with a fake problem: the measured step search, the
trust region and the learned-step accept rule (no GPU)."""
import numpy as np

from fwi3d_b200 import fwi, synth


class FakeProblem:
    """misfit(v) = |m - m*|^2 scaled, with m = 1/v^2 (a quadratic bowl)."""

    def __init__(self, v_true, v0):
        self.w = synth.Workload("fake", *v_true.shape[::-1], 10.0, 10, 1e-3, 30.0, 4, v_true,
                                np.zeros((1, 3)), np.zeros((1, 3)))
        self.mt = 1.0 / v_true.astype(np.float64) ** 2
        self.evals = 0
        self.gradients = 0
        self.vbounds = (0.0, np.inf)
        self.adopted = []

    def misfit(self, v):
        self.evals += 1
        m = 1.0 / v.astype(np.float64) ** 2
        return float(1e14 * np.sum((m - self.mt) ** 2))

    def adopt(self, v):
        self.adopted.append(fwi.model_key(v))

    def known_misfit(self, v):
        return self.misfit(v)

    def gradient(self, v):
        m = 1.0 / v.astype(np.float64) ** 2
        g = m - self.mt
        g = g / max(np.abs(g).max(), 1e-300)
        return g, g, np.ones_like(g), self.misfit(v)

    line_search = fwi.Fwi.line_search


def test_line_search_measures_the_step_it_returns():
    rng = np.random.default_rng(0)
    vt = rng.uniform(2000, 2200, (4, 5, 6)).astype(np.float32)
    v0 = np.full_like(vt, 2100.0)
    p = FakeProblem(vt, v0)
    dm = 1 / 2000.0 ** 2 - 1 / 2200.0 ** 2
    g, _, _, f0 = p.gradient(v0)
    v1, step, f1 = p.line_search(v0, g, f0, dm)
    assert 0 < step <= fwi.STEP_BOUND * 0.05 * dm
    assert f1 == p.misfit(v1) and f1 < f0  # the returned misfit is measured, not predicted
    assert p.adopted[-1] == fwi.model_key(v1)  # its residual is kept for the next gradient


def test_search_expands_while_the_misfit_falls_and_measures_the_vertex():
    a2 = 1.0
    calls = []

    def misfit(alpha, c):
        calls.append(alpha)
        return (alpha - c) ** 2 + 1.0

    def search(c):
        f0 = misfit(0.0, c)
        calls.clear()
        return fwi.search_step(lambda a: misfit(a, c), None, f0, 0.4, a2, 8.0)

    # minimum far beyond the trials: doubling up to the cap
    step, f = search(100.0)
    assert step == 8.0 and calls == [0.4, 1.0, 2.0, 4.0, 8.0]
    # minimum between two doublings: the parabola's vertex is measured and taken
    step, f = search(1.5)
    assert abs(step - 1.5) < 0.2 and calls[-1] == step and f == (step - 1.5) ** 2 + 1.0
    # every trial worse than no step: shrink, then give up
    step, f = search(-1.0)
    assert step == 0.0 and f == 2.0 and calls == [0.4, 1.0, 0.1, 0.025]


def test_step_is_bounded_by_the_trust_region():
    vt = np.full((3, 3, 3), 1500.0, np.float32)
    v0 = np.full_like(vt, 3000.0)  # far away: the misfit falls almost linearly
    p = FakeProblem(vt, v0)
    dm = 1 / 1500.0 ** 2 - 1 / 3000.0 ** 2
    g, _, _, f0 = p.gradient(v0)
    v1, step, _ = p.line_search(v0, g, f0, dm)
    assert step <= fwi.STEP_BOUND * 0.05 * dm * (1 + 1e-12)
    # no velocity moves by more than MAX_DV
    assert np.max(np.abs(v1.astype(np.float64) / v0 - 1.0)) <= fwi.MAX_DV * (1 + 1e-5)


def test_zero_or_non_finite_gradient_or_flat_model_gives_no_step():
    vt = np.full((2, 2, 2), 2000.0, np.float32)
    p = FakeProblem(vt, vt)
    for g, dm in ((np.zeros(vt.shape), 1e-7), (np.full(vt.shape, np.nan), 1e-7), (np.ones(vt.shape), 0.0)):
        v1, step, f = p.line_search(vt, g, 1.0, dm)
        assert step == 0.0 and f == 1.0 and np.array_equal(v1, vt)
    assert p.evals == 0


def test_learned_step_is_kept_only_when_its_measured_misfit_is_at_most_the_plain_one():
    rng = np.random.default_rng(1)
    vt = rng.uniform(2000, 2200, (4, 4, 4)).astype(np.float32)
    v0 = np.full_like(vt, 2100.0)
    good = lambda raw, v, ill: (vt - v).astype(np.float32)          # the exact update
    bad = lambda raw, v, ill: np.full_like(v, 300.0)                 # a harmful update
    quiet = lambda *a: None
    _, h_good = fwi.run(FakeProblem(vt, v0), v0, 2, learned=good, log=quiet)
    _, h_bad = fwi.run(FakeProblem(vt, v0), v0, 2, learned=bad, log=quiet)
    _, h_plain = fwi.run(FakeProblem(vt, v0), v0, 2, log=quiet)
    assert h_good[0]["choice"] == "learned" and h_good[-1]["misfit"] < 1e-6 * h_plain[-1]["misfit"]
    assert all(h["choice"] == "plain" for h in h_bad[:-1])
    assert h_bad[-1]["misfit"] == h_plain[-1]["misfit"]
    for h, nxt in zip(h_good[:-1], h_good[1:]):
        # the accept rule compares measured misfits, and the next iterate is the winner
        assert (h["choice"] == "learned") == (h["f_learned"] <= h["f_plain"])
        assert nxt["misfit"] == min(h["f_learned"], h["f_plain"])
