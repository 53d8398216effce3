"""Mixed-precision path (TF32 / BF16 tcgen05 trailing updates, FP64 diagonal
blocks, FP64 PCG refinement of alpha) against the FP64 numpy oracle.

Stated tolerances (error of this path, not of the reference):
  mean      : max|mu - mu_64| / max|mu_64|   <= 1e-8 (alpha refined in FP64)
  variance  : max|v - v_64| / v_64            <= 1.5e-2 (TF32), 5e-2 (BF16)
  NLML      : |l - l_64| / |l_64|             <= 1e-3 (TF32), 1e-2 (BF16)
(measured on this problem, whose smallest posterior variances are ~3e-3:
7.3e-3 and 2.1e-2 for the variance.)
The variance and the log-determinant carry the error of the low-precision
factor; alpha, and with it the mean and the data-fit term, are refined to a
1e-10 relative residual.
"""
import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu

VAR_TOL = {1: 1.5e-2, 2: 5e-2}
LOSS_TOL = {1: 1e-3, 2: 1e-2}


@pytest.fixture(scope="module")
def capi():
    from gprat_b200 import capi as c
    assert c.device_count() >= 1
    return c


@pytest.fixture(scope="module")
def problem():
    n, m, d, T = 2048, 512, 8, 256
    x, y, xt = O.synthetic(n, m, d)
    h = (1.0, 1.0, 0.1)
    o = O.OracleGP(x, y, n // T, T, d, h)
    om, ov = o.predict_with_uncertainty(xt, 1, m)
    return dict(n=n, m=m, d=d, T=T, x=x, y=y, xt=xt, h=h, om=om, ov=ov, loss=o.calculate_loss())


@pytest.mark.parametrize("prec", [1, 2])
def test_mixed_predictions(capi, problem, prec):
    p = problem
    gp = capi.CudaGP(p["x"], p["y"], p["n"] // p["T"], p["T"], p["d"])
    gp.set_precision(prec)
    mean, var = gp.predict_with_uncertainty(p["h"], p["xt"], 1, p["m"])
    mean_err = np.max(np.abs(mean - p["om"])) / np.max(np.abs(p["om"]))
    var_err = np.max(np.abs(var - p["ov"]) / p["ov"])
    loss = gp.compute_loss(p["h"])
    loss_err = abs(loss - p["loss"]) / abs(p["loss"])
    print(f"precision {prec}: mean err {mean_err:.3e}, var err {var_err:.3e}, loss err {loss_err:.3e}")
    assert mean_err <= 1e-8
    assert var_err <= VAR_TOL[prec]
    assert loss_err <= LOSS_TOL[prec]
    pm = gp.predict(p["h"], p["xt"], 1, p["m"])
    assert np.max(np.abs(pm - p["om"])) / np.max(np.abs(p["om"])) <= 1e-8


def test_mixed_matches_fp64_mode_of_same_library(capi, problem):
    p = problem
    gp = capi.CudaGP(p["x"], p["y"], p["n"] // p["T"], p["T"], p["d"])
    m64, v64 = gp.predict_with_uncertainty(p["h"], p["xt"], 1, p["m"])
    gp.set_precision(capi.PREC_MIXED_TF32)
    m32, v32 = gp.predict_with_uncertainty(p["h"], p["xt"], 1, p["m"])
    gp.set_precision(capi.PREC_FP64)
    m64b, _ = gp.predict_with_uncertainty(p["h"], p["xt"], 1, p["m"])
    assert np.array_equal(m64, m64b)  # switching modes leaves the FP64 path unchanged
    assert np.max(np.abs(m32 - m64)) / np.max(np.abs(m64)) <= 1e-8


def test_mixed_needs_multiple_of_128(capi):
    x, y, _ = O.synthetic(200, 8, 8)
    gp = capi.CudaGP(x, y, 2, 100, 8)
    with pytest.raises(capi.GpratCudaError) as e:
        gp.set_precision(capi.PREC_MIXED_TF32)
    assert e.value.code == capi.ERR_INVALID_ARG


def test_mixed_device_resident(capi, problem):
    import torch
    p = problem
    gp = capi.CudaGP(p["x"], p["y"], p["n"] // p["T"], p["T"], p["d"])
    gp.set_precision(capi.PREC_MIXED_BF16)
    dxt = torch.tensor(p["xt"], device="cuda")
    dm = torch.empty(p["m"], dtype=torch.float64, device="cuda")
    dv = torch.empty(p["m"], dtype=torch.float64, device="cuda")
    gp.fit_predict_device(p["h"], dxt.data_ptr(), dxt.numel(), p["m"], dm.data_ptr(), dv.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
    gp.check_status()
    mean, var = gp.predict_with_uncertainty(p["h"], p["xt"], 1, p["m"])
    assert np.allclose(dm.cpu().numpy(), mean, rtol=0, atol=1e-12 * np.max(np.abs(mean)))
    assert np.allclose(dv.cpu().numpy(), var, rtol=1e-12)


@pytest.mark.parametrize("prec", [1, 2])
def test_mixed_variance_recursive_solve(capi, problem, prec):
    """2560 test rows take the recursive-halving variance solve (512 rows take
    the 512-column panels); both meet the same stated tolerances, and the rows
    they share agree to the low-precision factor's error."""
    p = problem
    m2 = 2560
    _, _, xt2 = O.synthetic(p["n"], m2, p["d"])
    o = O.OracleGP(p["x"], p["y"], p["n"] // p["T"], p["T"], p["d"], p["h"])
    om2, ov2 = o.predict_with_uncertainty(xt2, 1, m2)
    gp = capi.CudaGP(p["x"], p["y"], p["n"] // p["T"], p["T"], p["d"])
    gp.set_precision(prec)
    mean2, var2 = gp.predict_with_uncertainty(p["h"], xt2, 1, m2)
    assert np.max(np.abs(mean2 - om2)) / np.max(np.abs(om2)) <= 1e-8
    assert np.max(np.abs(var2 - ov2) / ov2) <= VAR_TOL[prec]
    mean1, var1 = gp.predict_with_uncertainty(p["h"], xt2[: 512 + p["d"]], 1, 512)
    assert np.max(np.abs(var1 - var2[:512]) / ov2[:512]) <= VAR_TOL[prec]


@pytest.mark.parametrize("n", [128, 256, 384])
def test_mixed_overlapped_pipeline_small_factor(capi, n):
    """predict_with_uncertainty with 2048 test rows or more starts the variance
    solve beside the factorisation at fixed splits of the columns; with one to
    three 128-column blocks some of those ranges are empty."""
    m, d, T = 2048, 8, 128
    h = (1.0, 1.0, 0.1)
    x, y, xt = O.synthetic(n, m, d)
    o = O.OracleGP(x, y, n // T, T, d, h)
    om, ov = o.predict_with_uncertainty(xt, 1, m)
    gp = capi.CudaGP(x, y, n // T, T, d)
    gp.set_precision(capi.PREC_MIXED_TF32)
    mean, var = gp.predict_with_uncertainty(h, xt, 1, m)
    assert np.max(np.abs(mean - om)) / np.max(np.abs(om)) <= 1e-8
    assert np.max(np.abs(var - ov) / ov) <= VAR_TOL[1]
