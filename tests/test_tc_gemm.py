"""The tcgen05 tensor-core GEMM of the mixed-precision path, in isolation,
through its C-ABI test entry: C = beta*C + alpha*A B^T against an FP64 numpy
product.  Bound per element: the operand rounding of the kind (TF32: 2^-10
relative per operand, BF16: 2^-8) times sum_k |a_k b_k|, plus FP32
accumulation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {0: 4e-3, 1: 1.6e-2}  # per-element error / sum|a||b|


@pytest.fixture(scope="module")
def capi():
    from gprat_b200 import capi as c
    assert c.device_count() >= 1
    return c


def run_case(capi, kind, M, N, K, alpha, beta, lower=False, seed=0, with_rowsq=False, tile_mode=0):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = A.copy() if lower else rng.standard_normal((N, K)).astype(np.float32)
    C0 = rng.standard_normal((M, N)).astype(np.float32)
    C = C0.copy()
    rowsq = np.zeros(M) if with_rowsq else None
    capi.test_tc_gemm(kind, A, B, C, alpha, beta, lower, rowsq, tile_mode)
    prod = A.astype(np.float64) @ B.astype(np.float64).T
    want = beta * C0.astype(np.float64) + alpha * prod
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64).T + np.abs(C0) * beta + 1e-30
    err = np.abs(C - want) / scale
    if lower:
        il = np.tril_indices(M)
        assert np.max(err[il]) < TOL[kind]
        iu = np.triu_indices(M, 1)
        assert np.array_equal(C[iu], C0[iu]), "upper triangle must stay untouched"
    else:
        assert np.max(err) < TOL[kind]
    if with_rowsq:
        got = rowsq
        ref = np.sum(C.astype(np.float64) ** 2, axis=1)
        assert np.allclose(got, ref, rtol=1e-12)


@pytest.mark.parametrize("kind", [0, 1])
def test_square_update(capi, kind):
    run_case(capi, kind, 256, 256, 128, -1.0, 1.0)


@pytest.mark.parametrize("kind", [0, 1])
def test_overwrite_and_ragged_edges(capi, kind):
    run_case(capi, kind, 200, 130, 192, 1.0, 0.0, seed=1)


@pytest.mark.parametrize("kind", [0, 1])
def test_lower_triangle(capi, kind):
    run_case(capi, kind, 384, 384, 256, -1.0, 1.0, lower=True, seed=2)


def test_row_sums_of_squares(capi):
    run_case(capi, 0, 300, 128, 128, 1.0, 0.0, seed=3, with_rowsq=True)


@pytest.mark.parametrize("kind", [0, 1])
def test_persistent_multi_tile(capi, kind):
    # 16 x 16 tiles > 148 SMs: every CTA processes several tiles and both
    # TMEM accumulators
    run_case(capi, kind, 2048, 2048, 512, -1.0, 1.0, seed=4)


@pytest.mark.parametrize("kind", [0, 1])
def test_reduce_add_ragged_edges(capi, kind):
    # beta = 1 goes through the TMA reduce-add: partial tiles must be clipped
    run_case(capi, kind, 200, 130, 192, -1.0, 1.0, seed=5)
    run_case(capi, kind, 5, 7, 64, 1.0, 1.0, seed=6)


@pytest.mark.parametrize("kind", [0, 1])
def test_lower_triangle_ragged(capi, kind):
    run_case(capi, kind, 300, 300, 128, -1.0, 1.0, lower=True, seed=7)


@pytest.mark.parametrize("kind", [0, 1])
def test_wide_tiles(capi, kind):
    # N >= 512 runs the 128 x 256 tile: ragged edges, lower mode, both betas
    run_case(capi, kind, 700, 600, 128, 1.0, 0.0, seed=8)
    run_case(capi, kind, 1000, 1000, 192, -1.0, 1.0, lower=True, seed=9)
    run_case(capi, kind, 1536, 1536, 256, -1.0, 1.0, lower=True, seed=10)


@pytest.mark.parametrize("mode", [1, 2, 3])
@pytest.mark.parametrize("kind", [0, 1])
def test_every_tile_shape(capi, kind, mode):
    # the same cases through each tile shape: 128x128, 128x256, 256x256 on a CTA pair
    run_case(capi, kind, 640, 768, 128, 1.0, 0.0, seed=11, tile_mode=mode)
    run_case(capi, kind, 1000, 1000, 192, -1.0, 1.0, lower=True, seed=12, tile_mode=mode)
    run_case(capi, kind, 300, 520, 64, -1.0, 1.0, seed=13, tile_mode=mode)
    run_case(capi, kind, 2304, 2304, 256, -1.0, 1.0, lower=True, seed=14, tile_mode=mode)
