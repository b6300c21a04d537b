"""FWI driver on the GPU: the misfit of a model does not depend on what ran
before it (the line search and the accept rule compare misfits of models
built in different ways)."""
import numpy as np
import pytest

from fwi3d_b200 import fwi, synth

pytestmark = pytest.mark.gpu


def test_misfit_of_one_model_is_bit_reproducible():
    w = synth.small_fwi(0, n=40, nt=240)
    prob = fwi.Fwi(w, fwi.FwiOptions(batch=3, seed=5, rbc=w.rbc, zmask=w.zmask))
    f1 = prob.misfit(w.start)
    g, _, _, _ = prob.gradient(w.vp)          # other work on both contexts in between
    prob.misfit((w.start * 1.01).astype(np.float32))
    f2 = prob.misfit(w.start.copy())
    assert f1 == f2
    # a trial model reached through the line search's own arithmetic equals the
    # one rebuilt from the same step with a different scalar type
    dm = 1.0 / float(w.start.min()) ** 2 - 1.0 / float(w.start.max()) ** 2
    m = 1.0 / w.start.astype(np.float64) ** 2
    a = 0.05 * dm
    v_np = (1.0 / np.sqrt(m - np.float64(a) * np.asarray(g, np.float64))).astype(np.float32)
    v_py = (1.0 / np.sqrt(m - float(a) * np.asarray(g, np.float64))).astype(np.float32)
    assert np.array_equal(v_np, v_py)
    assert prob.misfit(v_np) == prob.misfit(v_py)
