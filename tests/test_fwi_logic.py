"""FWI driver logic on CPU with a fake problem: the bounded parabolic line
search and the learned-step accept rule (no GPU)."""
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

    def misfit(self, v):
        self.evals += 1
        m = 1.0 / v.astype(np.float64) ** 2
        return float(1e14 * np.sum((m - self.mt) ** 2))

    def gradient(self, v):
        m = 1.0 / v.astype(np.float64) ** 2
        g = m - self.mt
        g = g / max(np.abs(g).max(), 1e-300)
        return g, g, np.ones_like(g), self.misfit(v)

    line_search = fwi.Fwi.line_search


def test_line_search_finds_the_vertex_of_a_quadratic():
    rng = np.random.default_rng(0)
    vt = rng.uniform(2000, 2200, (4, 5, 6)).astype(np.float32)
    v0 = np.full_like(vt, 2100.0)
    p = FakeProblem(vt, v0)
    dm = 1 / 2000.0 ** 2 - 1 / 2200.0 ** 2
    g, _, _, f0 = p.gradient(v0)
    v1, step, pred = p.line_search(v0, g, f0, dm)
    assert 0 < step <= fwi.STEP_BOUND * 0.05 * dm
    assert p.misfit(v1) < f0
    assert p.evals == 4  # f0, two trial misfits and the check above


def test_step_is_bounded_when_the_parabola_extrapolates():
    vt = np.full((3, 3, 3), 1500.0, np.float32)
    v0 = np.full_like(vt, 3000.0)  # far away: the misfit falls almost linearly
    p = FakeProblem(vt, v0)
    dm = 1 / 1500.0 ** 2 - 1 / 3000.0 ** 2
    g, _, _, f0 = p.gradient(v0)
    v1, step, _ = p.line_search(v0, g, f0, dm)
    assert step <= fwi.STEP_BOUND * 0.05 * dm * (1 + 1e-12)
    # the trust region: no velocity moves by more than MAX_DV
    assert np.max(np.abs(v1.astype(np.float64) / v0 - 1.0)) <= fwi.MAX_DV * (1 + 1e-5)


def test_zero_or_non_finite_gradient_gives_no_step():
    vt = np.full((2, 2, 2), 2000.0, np.float32)
    p = FakeProblem(vt, vt)
    for g in (np.zeros(vt.shape), np.full(vt.shape, np.nan)):
        v1, step, pred = p.line_search(vt, g, 1.0, 1e-7)
        assert step == 0.0 and pred == 1.0 and np.array_equal(v1, vt)


def test_learned_step_is_kept_only_when_it_is_at_least_as_good():
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
