"""Per-phase step timers (gprat_cu_steps_*): the reference's APEX step labels,
timed with CUDA events around each phase of each call."""
import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu


def test_step_labels_and_times():
    from gprat_b200 import capi

    n, m, d, T = 1024, 256, 8, 128
    x, y, xt = O.synthetic(n, m, d)
    gp = capi.CudaGP(x, y, n // T, T, d)
    h = (1.0, 1.0, 0.1)
    capi.steps_reset()
    capi.steps_enable(True)
    try:
        gp.predict_with_uncertainty(h, xt, 1, m)
        gp.predict(h, xt, 1, m)
        gp.cholesky(h)
        gp.set_precision(capi.PREC_MIXED_TF32)
        gp.predict_with_uncertainty(h, xt, 1, m)
        st = capi.steps()
    finally:
        capi.steps_enable(False)
    for label in ("predict_uncer_step assembly", "predict_uncer_step cholesky", "predict_uncer_step forward",
                  "predict_uncer_step backward", "predict_uncer_step prediction", "predict_uncer_step forward KcK",
                  "predict_uncer_step prediction uncertainty", "predict_uncer_step alpha refinement",
                  "predict_step assembly", "predict_step prediction", "cholesky_step assembly",
                  "cholesky_step cholesky"):
        assert label in st, (label, sorted(st))
        calls, total = st[label]
        assert calls >= 1 and total > 0.0
    assert st["predict_uncer_step cholesky"][0] == 2  # FP64 and mixed calls
    capi.steps_reset()
    assert capi.steps() == {}
    # timers off: nothing recorded
    gp.predict(h, xt, 1, m)
    assert capi.steps() == {}
