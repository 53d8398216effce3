"""Parity of the CUDA path (through the C ABI) with the reference.

Golden sources: the reference's own known-answer file (data_1024/output.json,
tolerance of test/src/output_correctness.cpp: WithinRel 1e6*DBL_EPSILON), the
compiled reference's vectors in tests/golden/ref_cases.npz, and the numpy
oracle on seeded inputs at sizes it finishes in seconds.  FP64 bar: 1e-10
relative per element (mean, variance, L tiles) and for the loss.
"""
import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu

REL = 1e6 * np.finfo(float).eps  # 2.2e-10, the reference test's tolerance
FP64_TOL = 1e-10


@pytest.fixture(scope="module")
def capi():
    from gprat_b200 import capi as c
    assert c.device_count() >= 1
    return c


def rel_err(a, b, floor=1e-300):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


def test_known_answer_cholesky(capi, known_answer):
    g = known_answer
    T = g["n_train"] // g["n_tiles"]
    gp = capi.CudaGP(g["train_in"], g["train_out"], g["n_tiles"], T, g["n_reg"])
    tiles = gp.cholesky(g["kernel_params"])
    for got, want in zip(tiles, g["expected"]["choleksy"]):
        if len(want) == 0:
            assert got is None
        else:
            assert rel_err(got, want) <= REL


def test_known_answer_predictions(capi, known_answer):
    g = known_answer
    T = g["n_train"] // g["n_tiles"]
    mt, mts = O.compute_test_tiles(g["n_test"], g["n_tiles"], T)
    gp = capi.CudaGP(g["train_in"], g["train_out"], g["n_tiles"], T, g["n_reg"])
    h = g["kernel_params"]
    exp = g["expected"]
    mean, var = gp.predict_with_uncertainty(h, g["test_in"], mt, mts)
    assert rel_err(mean, exp["sum"][0]) <= REL and rel_err(var, exp["sum"][1]) <= REL
    mean, var = gp.predict_with_full_cov(h, g["test_in"], mt, mts)
    assert rel_err(mean, exp["full"][0]) <= REL and rel_err(var, exp["full"][1]) <= REL
    assert rel_err(gp.predict(h, g["test_in"], mt, mts), exp["pred"]) <= REL


def test_known_answer_optimize(capi, known_answer):
    g = known_answer
    T = g["n_train"] // g["n_tiles"]
    gp = capi.CudaGP(g["train_in"], g["train_out"], g["n_tiles"], T, g["n_reg"])
    lr, b1, b2, eps, it = g["adam"]
    params = np.array(list(g["kernel_params"]) + [0.0] * 6)
    losses, _ = gp.optimize(params, [lr, b1, b2, eps], [1, 1, 1], int(it))
    assert rel_err(losses, g["expected"]["losses"]) <= REL


@pytest.mark.parametrize("tag", ["c0", "ragged", "d64"])
def test_reference_vectors(capi, ref_cases, tag):
    n, m, d, T, mt, mts = (int(v) for v in ref_cases[f"{tag}_cfg"])
    h = ref_cases[f"{tag}_hyper"]
    x, y, xt = O.synthetic(n, m, d)
    gp = capi.CudaGP(x, y, n // T, T, d)
    mean, var = gp.predict_with_uncertainty(h, xt, mt, mts)
    assert rel_err(mean, ref_cases[f"{tag}_mean"]) < FP64_TOL
    assert rel_err(var, ref_cases[f"{tag}_var"]) < FP64_TOL
    fm, fv = gp.predict_with_full_cov(h, xt, mt, mts)
    assert rel_err(fv, ref_cases[f"{tag}_full_var"]) < FP64_TOL
    assert rel_err(gp.predict(h, xt, mt, mts), ref_cases[f"{tag}_pred"]) < FP64_TOL
    assert rel_err(gp.compute_loss(h), ref_cases[f"{tag}_loss"][0]) < FP64_TOL
    tiles = gp.cholesky(h)
    nt = n // T
    assert rel_err(tiles[0], ref_cases[f"{tag}_tile_0"]) < FP64_TOL
    assert rel_err(tiles[nt], ref_cases[f"{tag}_tile_10"], 1e-12) < FP64_TOL
    assert rel_err(tiles[nt * nt - 1], ref_cases[f"{tag}_tile_last"], 1e-12) < FP64_TOL


def test_reference_optimizer_trajectory(capi, ref_cases):
    n, d, T = (int(v) for v in ref_cases["opt_cfg"])
    x, y, _ = O.synthetic(n, 16, d)
    gp = capi.CudaGP(x, y, n // T, T, d)
    params = np.array([0.5, 2.0, 0.5] + [0.0] * 6)
    adam = [0.1, 0.9, 0.999, 1e-8]
    for it in range(5):
        _, g = gp.loss_grad(params[:3])
        assert rel_err(g, ref_cases["opt_grads"][it]) < FP64_TOL
        loss, params = gp.optimize_step(params, adam, [1, 1, 1], it)
        assert rel_err(loss, ref_cases["opt_losses"][it]) < FP64_TOL
        assert rel_err(params, ref_cases["opt_params"][it]) < FP64_TOL


def test_gradient_matches_central_differences(capi):
    n, d, T = 512, 8, 128
    x, y, _ = O.synthetic(n, 16, d)
    gp = capi.CudaGP(x, y, n // T, T, d)
    theta = np.array([0.7, 1.5, 0.3])
    _, g = gp.loss_grad(theta)
    h = 1e-6
    for q in range(3):
        noise = q == 2
        u = O.to_unconstrained(theta[q], noise)
        tp, tm = theta.copy(), theta.copy()
        tp[q] = O.to_constrained(u + h, noise)
        tm[q] = O.to_constrained(u - h, noise)
        fd = (gp.compute_loss(tp) - gp.compute_loss(tm)) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q]))


@pytest.mark.parametrize("n,m,T,d", [(1000, 300, 100, 8), (2048, 512, 256, 8), (384, 100, 96, 3),
                                     (1000, 300, 100, 16), (1536, 257, 128, 40), (700, 130, 70, 100)])
def test_against_numpy_oracle(capi, n, m, T, d):
    x, y, xt = O.synthetic(n, m, d)
    h = (1.3, 0.8, 0.05)
    gp = capi.CudaGP(x, y, n // T, T, d)
    o = O.OracleGP(x, y, n // T, T, d, h)
    mean, var = gp.predict_with_uncertainty(h, xt, 1, m)
    om, ov = o.predict_with_uncertainty(xt, 1, m)
    assert rel_err(mean, om, 1e-12) < FP64_TOL
    assert rel_err(var, ov) < FP64_TOL
    assert rel_err(gp.compute_loss(h), o.calculate_loss()) < FP64_TOL


def test_full_posterior_covariance(capi):
    n, m, d, T = 512, 96, 8, 128
    x, y, xt = O.synthetic(n, m, d)
    h = (1.0, 1.0, 0.1)
    gp = capi.CudaGP(x, y, n // T, T, d)
    mean, cov = gp.predict_full_covariance(h, xt, m)
    o = O.OracleGP(x, y, n // T, T, d, h)
    want = o.posterior_covariance(xt, m)
    assert np.max(np.abs(cov - want)) < 1e-10 * np.max(np.abs(want))
    _, var = gp.predict_with_uncertainty(h, xt, 1, m)
    assert rel_err(np.diag(cov), var) < 1e-9


def test_not_positive_definite_is_reported(capi):
    x, y, _ = O.synthetic(256, 8, 8)
    gp = capi.CudaGP(x, y, 2, 128, 8)
    with pytest.raises(capi.NotPositiveDefiniteError):
        gp.compute_loss((1.0, 1.0, -5.0))
    # the handle stays usable afterwards
    assert np.isfinite(gp.compute_loss((1.0, 1.0, 0.1)))


def test_empty_test_set(capi):
    x, y, _ = O.synthetic(256, 8, 8)
    gp = capi.CudaGP(x, y, 2, 128, 8)
    mean, var = gp.predict_with_uncertainty((1.0, 1.0, 0.1), np.zeros(7), 0, 0)
    assert mean.size == 0 and var.size == 0


def test_device_resident_fit_predict(capi):
    import torch
    n, m, d, T = 1024, 512, 8, 128
    x, y, xt = O.synthetic(n, m, d)
    h = (1.0, 1.0, 0.1)
    gp = capi.CudaGP(x, y, n // T, T, d)
    dxt = torch.tensor(xt, device="cuda")
    dmean = torch.empty(m, dtype=torch.float64, device="cuda")
    dvar = torch.empty(m, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    gp.fit_predict_device(h, dxt.data_ptr(), dxt.numel(), m, dmean.data_ptr(), dvar.data_ptr(), stream.cuda_stream)
    gp.check_status()
    mean, var = gp.predict_with_uncertainty(h, xt, 1, m)
    assert np.array_equal(dmean.cpu().numpy(), mean)
    assert np.array_equal(dvar.cpu().numpy(), var)
