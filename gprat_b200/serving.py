"""Serving front end over the C ABI's gprat_cu_server_* and
gprat_cu_multiserver_* entry points.

A :class:`Server` keeps fitted GP models resident on one GPU (factor and
weights stay in HBM) and answers asynchronous predict and fit requests.  A
:class:`MultiServer` replicates every model on several GPUs and spreads the
predict requests over them.  The batching, scheduling, memory admission and
replica routing run natively in the library (gprat_b200/csrc/serve.cu,
multiserve.cu); this module only marshals arrays.  There is no
counterpart in the reference, whose predict calls re-factorise the training
covariance every time (core/src/cpu/gp_functions.cpp:110-189).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import numpy as np

from . import capi

_dp = ctypes.POINTER(ctypes.c_double)


@dataclass
class ServerStats:
    p50_ms: float
    p99_ms: float
    predictions_per_s: float
    completed: int
    batches: int


class Server:
    """Resident-model GP server on one device.

    precision: ``capi.PREC_FP64`` / ``PREC_MIXED_TF32`` / ``PREC_MIXED_BF16``
    for every model of the server.  memory_budget_bytes <= 0 takes 80 % of the
    device memory free at creation.
    """

    _PREFIX = "gprat_cu_server_"

    def __init__(self, device: int = 0, memory_budget_bytes: int = 0, precision: int = capi.PREC_FP64):
        h = ctypes.c_void_p()
        capi.check(capi.lib.gprat_cu_server_create(int(device), int(memory_budget_bytes), int(precision),
                                                   ctypes.byref(h)))
        self._init_handle(h)

    def _init_handle(self, h: ctypes.c_void_p) -> None:
        self._h = h
        self._m = {}      # request id -> number of test points (0 for fits)
        self._reg = {}    # model id -> regressors

    def _fn(self, name: str):
        return getattr(capi.lib, self._PREFIX + name)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            capi.check(self._fn("destroy")(self._h))
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_model(self, x: Sequence[float], y: Sequence[float], n_tiles: int, n_tile_size: int, n_reg: int,
                  hyper) -> int:
        """Fits a model synchronously; returns its id."""
        x, y, hy = capi._arr(x), capi._arr(y), capi._hyper(hyper)
        mid = ctypes.c_int()
        capi.check(self._fn("add_model")(self._h, capi._p(x), x.size, capi._p(y), y.size, int(n_tiles),
                                                      int(n_tile_size), int(n_reg), capi._p(hy), ctypes.byref(mid)))
        self._reg[mid.value] = int(n_reg)
        return mid.value

    def submit_predict(self, model_id: int, xt: Sequence[float], m: Optional[int] = None) -> int:
        """Queues m test points (sliding windows over xt); returns a request id."""
        xt = capi._arr(xt)
        if m is None:
            m = xt.size - self._reg.get(model_id, 1) + 1
        rid = ctypes.c_int64()
        capi.check(self._fn("submit_predict")(self._h, int(model_id), capi._p(xt), xt.size, int(m),
                                                           ctypes.byref(rid)))
        self._m[rid.value] = int(m)
        return rid.value

    def submit_fit(self, x: Sequence[float], y: Sequence[float], n_tiles: int, n_tile_size: int, n_reg: int,
                   hyper) -> int:
        """Queues the fit of a new model; wait() on the id returns the model id."""
        x, y, hy = capi._arr(x), capi._arr(y), capi._hyper(hyper)
        rid = ctypes.c_int64()
        capi.check(self._fn("submit_fit")(self._h, capi._p(x), x.size, capi._p(y), y.size, int(n_tiles),
                                                       int(n_tile_size), int(n_reg), capi._p(hy), ctypes.byref(rid)))
        self._m[rid.value] = 0
        self._reg[("fit", rid.value)] = int(n_reg)
        return rid.value

    def wait(self, request_id: int) -> Tuple[Optional[np.ndarray], Optional[np.ndarray], int, float]:
        """Blocks until the request is done: (mean, var, model_id, latency_ms).

        mean and var are None for fit requests."""
        m = self._m.pop(request_id, 0)
        mean = np.empty(m) if m else None
        var = np.empty(m) if m else None
        mid = ctypes.c_int()
        lat = ctypes.c_double()
        capi.check(self._fn("wait")(self._h, int(request_id), capi._p(mean) if m else None,
                                                 capi._p(var) if m else None, ctypes.byref(mid), ctypes.byref(lat)))
        n_reg = self._reg.pop(("fit", request_id), None)
        if n_reg is not None:
            self._reg[mid.value] = n_reg
        return mean, var, mid.value, lat.value

    def stats(self) -> ServerStats:
        p50, p99, pps = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        done, batches = ctypes.c_int64(), ctypes.c_int64()
        capi.check(self._fn("stats")(self._h, ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(pps),
                                                  ctypes.byref(done), ctypes.byref(batches)))
        return ServerStats(p50.value, p99.value, pps.value, done.value, batches.value)


class MultiServer(Server):
    """Replica serving over several devices (one server per entry of
    ``devices``; a device may repeat).  Every model is fitted on each replica
    and keeps one model id; a predict request goes to the replica with the
    fewest test points outstanding and its result is bit-identical to the same
    request on a single :class:`Server`.  replication: ``capi.REPLICATE_COPY``
    fits a model on the first replica and copies its fitted state to the
    others (peer copies); ``capi.REPLICATE_REFIT`` fits it on every replica at
    once.  memory_budget_bytes and precision apply to each replica."""

    _PREFIX = "gprat_cu_multiserver_"

    def __init__(self, devices: Sequence[int] = (0,), memory_budget_bytes: int = 0,
                 precision: int = capi.PREC_FP64, replication: int = capi.REPLICATE_COPY):
        devs = (ctypes.c_int * len(devices))(*[int(d) for d in devices])
        h = ctypes.c_void_p()
        capi.check(capi.lib.gprat_cu_multiserver_create(devs, len(devices), int(memory_budget_bytes),
                                                        int(precision), ctypes.byref(h)))
        self.n_replicas = len(devices)
        self._init_handle(h)
        capi.check(capi.lib.gprat_cu_multiserver_set_replication(self._h, int(replication)))

    def replica_completed(self) -> list:
        """Predict requests waited on, per replica that served them."""
        out = []
        for r in range(self.n_replicas):
            c = ctypes.c_int64()
            capi.check(capi.lib.gprat_cu_multiserver_replica_completed(self._h, r, ctypes.byref(c)))
            out.append(c.value)
        return out

    def resident_bytes(self) -> list:
        """Device bytes the resident models hold, per replica."""
        out = []
        for r in range(self.n_replicas):
            c = ctypes.c_int64()
            capi.check(capi.lib.gprat_cu_multiserver_resident_bytes(self._h, r, ctypes.byref(c)))
            out.append(c.value)
        return out

    def fail_next_copy(self, replica: int) -> None:
        """Test hook: the next copy of a fitted model to `replica` fails (on the host)."""
        capi.check(capi.lib.gprat_cu_test_multiserver_fail_copy(self._h, int(replica)))
