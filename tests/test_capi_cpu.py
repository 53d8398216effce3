"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/gprat_cu.h declares, and rejects bad arguments before touching the
device.  No compute call is made here."""
import ctypes
import subprocess

import numpy as np
import pytest

from gprat_b200 import capi


def test_library_exports_every_declared_symbol():
    declared = capi.declared_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(capi.lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in capi.lib.gprat_cu_version()


def test_device_count_never_fails():
    assert capi.device_count() >= 0


def test_create_rejects_short_series():
    x = np.zeros(10)
    y = np.zeros(16)
    with pytest.raises(capi.GpratCudaError) as e:
        capi.CudaGP(x, y, 4, 4, 8)
    assert e.value.code == capi.ERR_INVALID_ARG
    assert "sliding window" in str(e.value)


def test_create_rejects_short_outputs():
    with pytest.raises(capi.GpratCudaError) as e:
        capi.CudaGP(np.zeros(64), np.zeros(8), 4, 4, 8)
    assert e.value.code == capi.ERR_INVALID_ARG


def test_create_rejects_bad_tiling():
    with pytest.raises(capi.GpratCudaError) as e:
        capi.CudaGP(np.zeros(64), np.zeros(64), 0, 4, 8)
    assert e.value.code == capi.ERR_INVALID_ARG


def test_null_handle_is_rejected():
    h = np.array([1.0, 1.0, 0.1])
    v = ctypes.c_double()
    rc = capi.lib.gprat_cu_compute_loss(None, h.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(v))
    assert rc == capi.ERR_INVALID_ARG
    assert b"NULL" in capi.lib.gprat_cu_last_error()


def test_multiserver_rejects_empty_device_list():
    from gprat_b200 import serving
    with pytest.raises(capi.GpratCudaError) as e:
        serving.MultiServer([])
    assert e.value.code == capi.ERR_INVALID_ARG


def test_multiserver_without_a_device():
    if capi.device_count() > 0:
        pytest.skip("a GPU is visible")
    from gprat_b200 import serving
    with pytest.raises(capi.GpratCudaError) as e:
        serving.MultiServer([0, 0])
    assert e.value.code == capi.ERR_NO_DEVICE


def test_multiserver_null_handle_is_rejected():
    v = ctypes.c_int64()
    assert capi.lib.gprat_cu_multiserver_wait(None, 1, None, None, None, None) == capi.ERR_INVALID_ARG
    assert capi.lib.gprat_cu_multiserver_set_replication(None, capi.REPLICATE_COPY) == capi.ERR_INVALID_ARG
    assert capi.lib.gprat_cu_multiserver_replica_completed(None, 0, ctypes.byref(v)) == capi.ERR_INVALID_ARG
    assert capi.lib.gprat_cu_multiserver_destroy(None) == capi.OK


def test_trsv_entry_rejects_bad_arguments():
    L = np.eye(4)
    with pytest.raises(capi.GpratCudaError) as e:
        capi.test_trsv(2, L, np.ones(4))  # no such kind
    assert e.value.code == capi.ERR_INVALID_ARG


def test_mode_setters_reject_a_null_handle():
    """The precision-mode setters, the CG counter and the device-resident call
    validate the handle before anything reaches the device."""
    lib = capi.lib
    calls = [
        lambda: lib.gprat_cu_gp_set_precision(None, capi.PREC_FP64_INT8),
        lambda: lib.gprat_cu_gp_set_int8_slices(None, 5),
        lambda: lib.gprat_cu_gp_set_int8_groups(None, 4, 4),
        lambda: lib.gprat_cu_gp_pcg_iterations(None, ctypes.byref(ctypes.c_int())),
    ]
    for call in calls:
        assert call() == capi.ERR_INVALID_ARG
        assert b"NULL" in lib.gprat_cu_last_error()
    h = np.array([1.0, 1.0, 0.1])
    rc = lib.gprat_cu_fit_predict_device(None, h.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None, 0, 0,
                                         None, None, None)
    assert rc == capi.ERR_INVALID_ARG
