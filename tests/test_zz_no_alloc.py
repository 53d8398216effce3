"""The allocation-free loss entry point (gprat_cu_compute_loss_noalloc).

Callers that cannot call cudaMalloc -- code running under an allocator or a
memory pool it does not own, or a latency-critical loop that must not enter
the driver's allocator -- use this entry point with their own device buffers;
its scratch is a fixed device array inside the library.  This test calls it
through the C ABI and checks that it returns the same loss as the regular
entry point (gprat_cu_compute_loss) and as the numpy oracle on two calls in a
row, at the FP64 tolerance of the other GPU tests: at the size limit (1024
training points), with a ragged last block (300 points in tiles of 100), and
after a call that fails on a covariance that is not positive definite (the
shared status word must start clean again).  The file name makes pytest
collect it last; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _bind(lib):
    dp = ctypes.POINTER(ctypes.c_double)
    f = lib.gprat_cu_compute_loss_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                  ctypes.c_int, ctypes.c_int, dp, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _call(f, dx, dy, n_tiles, T, d, hyper, dloss, stream):
    h = np.array(hyper, dtype=np.float64)
    return f(0, dx.data_ptr(), dx.numel(), dy.data_ptr(), dy.numel(), n_tiles, T, d,
             h.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), dloss.data_ptr(), stream)


@pytest.mark.parametrize("n,T", [(1000, 125), (1024, 128), (300, 100)])
def test_noalloc_loss_matches_regular_entry_point(n, T):
    import torch

    from gprat_b200 import capi

    f = _bind(capi.lib)
    d = 8
    x, y, _ = O.synthetic(n, 8, d)
    dx = torch.tensor(x, device="cuda")
    dy = torch.tensor(y, device="cuda")
    dloss = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    gp = capi.CudaGP(x, y, n // T, T, d)
    stream = torch.cuda.current_stream().cuda_stream
    for hyper in ((1.0, 1.0, 0.1), (0.6, 1.7, 0.05)):
        rc = _call(f, dx, dy, n // T, T, d, hyper, dloss, stream)
        assert rc == capi.OK, capi.lib.gprat_cu_last_error().decode()
        got = float(dloss.item())
        want = gp.compute_loss(hyper)
        oracle = O.OracleGP(x, y, n // T, T, d, hyper).calculate_loss()
        assert abs(got - want) <= FP64_TOL * abs(want)
        assert abs(got - oracle) <= FP64_TOL * abs(oracle)
    gp.close()


def test_noalloc_not_positive_definite_then_clean():
    import torch

    from gprat_b200 import capi

    f = _bind(capi.lib)
    n, d, T = 512, 8, 128
    x, y, _ = O.synthetic(n, 8, d)
    dx = torch.tensor(x, device="cuda")
    dy = torch.tensor(y, device="cuda")
    dloss = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = _call(f, dx, dy, n // T, T, d, (1.0, 1.0, -5.0), dloss, stream)
    assert rc == capi.ERR_NOT_SPD
    assert b"positive definite" in capi.lib.gprat_cu_last_error()
    rc = _call(f, dx, dy, n // T, T, d, (1.0, 1.0, 0.1), dloss, stream)
    assert rc == capi.OK, capi.lib.gprat_cu_last_error().decode()
    want = O.OracleGP(x, y, n // T, T, d, (1.0, 1.0, 0.1)).calculate_loss()
    assert abs(float(dloss.item()) - want) <= FP64_TOL * abs(want)


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch

    from gprat_b200 import capi

    f = _bind(capi.lib)
    n, d = 2048, 8
    dx = torch.zeros(n + d, dtype=torch.float64, device="cuda")
    dy = torch.zeros(n, dtype=torch.float64, device="cuda")
    dloss = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _call(f, dx, dy, 16, 128, d, (1.0, 1.0, 0.1), dloss, None)
    assert rc == capi.ERR_INVALID_ARG
    assert b"limit" in capi.lib.gprat_cu_last_error()
