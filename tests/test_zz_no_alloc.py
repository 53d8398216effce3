"""The allocation-free loss entry point (gprat_cu_compute_loss_noalloc).

Callers that cannot call cudaMalloc -- code running under an allocator or a
memory pool it does not own, or a latency-critical loop that must not enter
the driver's allocator -- use this entry point with their own device buffers;
its scratch is a fixed device array inside the library.  This test calls it
through the C ABI and checks that it returns the same loss as the regular
entry point (gprat_cu_compute_loss) on two calls in a row, at the FP64
tolerance of the other GPU tests.  The file name makes pytest collect it
last; it also passes alone in a fresh process.
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


def test_noalloc_loss_matches_regular_entry_point():
    import torch

    from gprat_b200 import capi

    f = _bind(capi.lib)
    n, d, T = 1000, 8, 125
    x, y, _ = O.synthetic(n, 8, d)
    dx = torch.tensor(x, device="cuda")
    dy = torch.tensor(y, device="cuda")
    dloss = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    gp = capi.CudaGP(x, y, n // T, T, d)
    stream = torch.cuda.current_stream().cuda_stream
    for hyper in ((1.0, 1.0, 0.1), (0.6, 1.7, 0.05)):
        h = np.array(hyper)
        rc = f(0, dx.data_ptr(), dx.numel(), dy.data_ptr(), dy.numel(), n // T, T, d,
               h.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), dloss.data_ptr(), stream)
        assert rc == capi.OK, capi.lib.gprat_cu_last_error().decode()
        got = float(dloss.item())
        want = gp.compute_loss(hyper)
        assert abs(got - want) <= FP64_TOL * abs(want)


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch

    from gprat_b200 import capi

    f = _bind(capi.lib)
    n, d = 2048, 8
    dx = torch.zeros(n + d, dtype=torch.float64, device="cuda")
    dy = torch.zeros(n, dtype=torch.float64, device="cuda")
    dloss = torch.zeros(1, dtype=torch.float64, device="cuda")
    h = np.array([1.0, 1.0, 0.1])
    rc = f(0, dx.data_ptr(), dx.numel(), dy.data_ptr(), dy.numel(), 16, 128, d,
           h.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), dloss.data_ptr(), None)
    assert rc == capi.ERR_INVALID_ARG
    assert b"limit" in capi.lib.gprat_cu_last_error()
