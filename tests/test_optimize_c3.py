"""Hyper-parameter optimisation at n_train = 8192 (d = 8, 16 x 16 tiles of
512; initial lengthscale 0.5, vertical_lengthscale 2.0, noise 0.5; 50 Adam
steps at lr = 0.1, beta1 = 0.9, beta2 = 0.999) in FP64 with the adjoint
kernel, against the reference's own CPU trajectory (tests/golden/c3_optimize.npz,
made by tests/golden/make_golden.py --c3):

* loss and parameters after every step: 1e-10 relative;
* gradient at steps 0, 10, 20, 30, 40: 1e-9 relative to the reference's, and
  1e-6 relative to central differences of the library's loss (h = 1e-6 in the
  unconstrained parameter, as the gradient is defined).
"""
import os

import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c3_optimize.npz")


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


@pytest.fixture(scope="module")
def c3():
    if not os.path.exists(GOLDEN):
        pytest.skip("c3_optimize.npz not generated")
    return np.load(GOLDEN)


def test_adam_trajectory_and_gradients(c3):
    from gprat_b200 import capi

    n, d, T, steps = (int(v) for v in c3["cfg"])
    adam = list(c3["adam"])
    checkpoints = list(c3["checkpoints"])
    x, y, _ = O.synthetic(n, 16, d)
    gp = capi.CudaGP(x, y, n // T, T, d)
    params = np.array([0.5, 2.0, 0.5] + [0.0] * 6)
    ci = 0
    for it in range(steps):
        if it in checkpoints:
            loss0, g = gp.loss_grad(params[:3])
            assert rel(g, c3["grads"][ci]) < 1e-9, (it, g, c3["grads"][ci])
            h = 1e-6
            for q in range(3):
                noise = q == 2
                u = O.to_unconstrained(params[q], noise)
                tp, tm = params[:3].copy(), params[:3].copy()
                tp[q] = O.to_constrained(u + h, noise)
                tm[q] = O.to_constrained(u - h, noise)
                fd = (gp.compute_loss(tp) - gp.compute_loss(tm)) / (2 * h)
                assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q])), (it, q, fd, g[q])
            ci += 1
        loss, params = gp.optimize_step(params, adam, [1, 1, 1], it)
        assert rel(loss, c3["losses"][it]) < 1e-10, (it, loss, c3["losses"][it])
        assert rel(params, c3["params"][it]) < 1e-10, (it, params, c3["params"][it])
