"""Bounded device waits: the single-launch triangular solves wait for earlier
row blocks by re-reading x (a sentinel marks unsolved entries).  With the
poll budget shrunk to 0 (gprat_cu_test_set_wait_budget), a wait on an
unsolved block gives up at once: the kernel sets the status word's timeout
flag and finishes, and the call returns GPRAT_CU_ERR_TIMEOUT.  With the
default budget restored, the same handle solves correctly again.  Only global
memory is polled, so nothing is left in flight when a wait gives up.
"""
import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from gprat_b200 import capi as c

    assert c.device_count() >= 1
    return c


def test_forced_expiry_then_recovery(capi):
    n, m, d, T = 4096, 256, 8, 256
    h = (1.0, 1.0, 0.1)
    x, y, xt = O.synthetic(n, m, d)
    gp = capi.CudaGP(x, y, n // T, T, d)
    try:
        capi.test_set_wait_budget(0)
        with pytest.raises(capi.GpratCudaError) as err:
            gp.predict_with_uncertainty(h, xt, 1, m)
        assert err.value.code == capi.ERR_TIMEOUT
        L = np.tril(np.linalg.cholesky(O.covariance(x, n, d, h)))
        b = np.random.default_rng(3).standard_normal(n)
        with pytest.raises(capi.GpratCudaError) as err:
            capi.test_trsv(0, L, b)
        assert err.value.code == capi.ERR_TIMEOUT
    finally:
        capi.test_set_wait_budget(-1)
    mean, var = gp.predict_with_uncertainty(h, xt, 1, m)
    om, ov = O.OracleGP(x, y, n // T, T, d, h).predict_with_uncertainty(xt, 1, m)
    assert np.max(np.abs(mean - om)) / np.max(np.abs(om)) <= 1e-10
    assert np.max(np.abs(var - ov) / ov) <= 1e-10
    gp.close()
