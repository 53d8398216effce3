"""Single-launch blocked triangular solves (trsv_fused.cu) against numpy.

The FP64 kernels carry the FP64 alpha solve (forward_solve_tiled /
backward_solve_tiled, core/src/cpu/tiled_algorithms.cpp:61-115); the FP32
ones are the preconditioner of the mixed path's refinement, whose last two
products per row block round to FP32.  Sizes cover one block, a ragged last
block and a few hundred blocks; max_ctas > 0 makes every CTA take several
row blocks by ticket.
"""
import numpy as np
import pytest
from scipy.linalg import solve_triangular

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from gprat_b200 import capi
    assert capi.device_count() >= 1
    return capi


def _factor(n, seed):
    rng = np.random.default_rng(seed)
    L = np.tril(rng.standard_normal((n, n))) / np.sqrt(n)
    L[np.diag_indices(n)] = rng.uniform(1.0, 2.0, n)
    return L


@pytest.mark.parametrize("n,max_ctas", [(128, 0), (1000, 0), (1000, 3), (4160, 0), (4160, 7), (33 * 128, 148)])
def test_fp64_solves(capi, n, max_ctas):
    L = _factor(n, n)
    b = np.random.default_rng(1).standard_normal(n)
    xf, xb = capi.test_trsv(0, L, b, max_ctas)
    ef = solve_triangular(L, b, lower=True)
    eb = solve_triangular(L.T, b, lower=False)
    assert np.max(np.abs(xf - ef)) <= 1e-12 * np.max(np.abs(ef))
    assert np.max(np.abs(xb - eb)) <= 1e-12 * np.max(np.abs(eb))


@pytest.mark.parametrize("n,max_ctas", [(128, 0), (200, 0), (1000, 0), (1000, 3), (4160, 0), (4160, 7),
                                        (8192, 0), (8192, 148)])
def test_fp32_solves(capi, n, max_ctas):
    L = _factor(n, n + 7)
    b = np.random.default_rng(2).standard_normal(n)
    xf, xb = capi.test_trsv(1, L, b, max_ctas)
    # against the exact solve with the FP32-rounded factor: what is left is the
    # kernels' own arithmetic (FP32 rounding of the last two products per block)
    L32 = L.astype(np.float32).astype(np.float64)
    ef = solve_triangular(L32, b, lower=True)
    eb = solve_triangular(L32.T, b, lower=False)
    assert np.max(np.abs(xf - ef)) <= 2e-5 * np.max(np.abs(ef))
    assert np.max(np.abs(xb - eb)) <= 2e-5 * np.max(np.abs(eb))
