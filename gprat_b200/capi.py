"""ctypes binding of the C ABI in include/gprat_cu.h (libgprat_cuda.so).

This is the thinnest host path to the CUDA kernels: tests and the benchmark
call the library through it exactly as a foreign-language caller would.  The
library must have been built (``python -m gprat_b200.build``); importing this
module fails loudly otherwise -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re
from typing import List, Optional, Sequence, Tuple

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libgprat_cuda.so")
HEADER = os.path.join(os.path.dirname(_PKG), "include", "gprat_cu.h")

OK = 0
ERR_INVALID_ARG = 1
ERR_OOM = 2
ERR_NOT_SPD = 3
ERR_CUDA = 4
ERR_TIMEOUT = 5
ERR_NO_DEVICE = 6

PREC_FP64 = 0
PREC_MIXED_TF32 = 1
PREC_MIXED_BF16 = 2
PREC_FP64_INT8 = 3  # FP64 data, every product emulated on the int8 tensor cores (Ozaki scheme)

REPLICATE_COPY = 0
REPLICATE_REFIT = 1


class GpratCudaError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[gprat_cu error {code}] {message}")
        self.code = code


class NotPositiveDefiniteError(GpratCudaError):
    pass


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_i64 = ctypes.c_int64


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libgprat_cuda.so is not built ({LIB_PATH}); run `python -m gprat_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    lib.gprat_cu_last_error.restype = ctypes.c_char_p
    lib.gprat_cu_version.restype = ctypes.c_char_p
    lib.gprat_cu_device_count.argtypes = [_ip]
    lib.gprat_cu_gp_create.argtypes = [ctypes.c_int, _dp, _i64, _dp, _i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_void_p)]
    lib.gprat_cu_gp_destroy.argtypes = [ctypes.c_void_p]
    lib.gprat_cu_gp_set_precision.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.gprat_cu_gp_set_int8_slices.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.gprat_cu_gp_set_int8_groups.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    lib.gprat_cu_cholesky.argtypes = [ctypes.c_void_p, _dp, _dp]
    lib.gprat_cu_predict.argtypes = [ctypes.c_void_p, _dp, _dp, _i64, ctypes.c_int, ctypes.c_int, _dp]
    for name in ("gprat_cu_predict_with_uncertainty", "gprat_cu_predict_with_full_cov"):
        getattr(lib, name).argtypes = [ctypes.c_void_p, _dp, _dp, _i64, ctypes.c_int, ctypes.c_int, _dp, _dp]
    lib.gprat_cu_predict_full_covariance.argtypes = [ctypes.c_void_p, _dp, _dp, _i64, ctypes.c_int, _dp, _dp]
    lib.gprat_cu_compute_loss.argtypes = [ctypes.c_void_p, _dp, _dp]
    lib.gprat_cu_loss_grad.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
    lib.gprat_cu_optimize_step.argtypes = [ctypes.c_void_p, _dp, _dp, _ip, ctypes.c_int, _dp]
    lib.gprat_cu_optimize.argtypes = [ctypes.c_void_p, _dp, _dp, _ip, ctypes.c_int, _dp]
    lib.gprat_cu_fit_predict_device.argtypes = [ctypes.c_void_p, _dp, ctypes.c_void_p, _i64, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.gprat_cu_check_status.argtypes = [ctypes.c_void_p]
    lib.gprat_cu_gp_pcg_iterations.argtypes = [ctypes.c_void_p, _ip]
    lib.gprat_cu_stats_enable_timing.argtypes = [ctypes.c_int]
    lib.gprat_cu_stats_read.argtypes = [ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), _dp, _dp]
    _fp = ctypes.POINTER(ctypes.c_float)
    lib.gprat_cu_test_tc_gemm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _fp, _i64, _fp,
                                          _i64, _fp, _i64, ctypes.c_float, ctypes.c_float, ctypes.c_int, _dp,
                                          ctypes.c_int]
    _vp, _i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)
    lib.gprat_cu_steps_enable.argtypes = [ctypes.c_int]
    lib.gprat_cu_test_trsv.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int]
    lib.gprat_cu_test_set_wait_budget.argtypes = [_i64]
    _i8p, _i32p = ctypes.POINTER(ctypes.c_int8), ctypes.POINTER(ctypes.c_int32)
    lib.gprat_cu_test_oz_split.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, _i8p, _i32p]
    lib.gprat_cu_test_oz_gemm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                          ctypes.c_int]
    lib.gprat_cu_steps_csv.argtypes = [ctypes.c_char_p, _i64, _i64p]
    lib.gprat_cu_server_create.argtypes = [ctypes.c_int, _i64, ctypes.c_int, ctypes.POINTER(_vp)]
    lib.gprat_cu_server_destroy.argtypes = [_vp]
    lib.gprat_cu_server_add_model.argtypes = [_vp, _dp, _i64, _dp, _i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              _dp, _ip]
    lib.gprat_cu_server_submit_predict.argtypes = [_vp, ctypes.c_int, _dp, _i64, ctypes.c_int, _i64p]
    lib.gprat_cu_server_submit_fit.argtypes = [_vp, _dp, _i64, _dp, _i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               _dp, _i64p]
    lib.gprat_cu_server_wait.argtypes = [_vp, _i64, _dp, _dp, _ip, _dp]
    lib.gprat_cu_server_stats.argtypes = [_vp, _dp, _dp, _dp, _i64p, _i64p]
    lib.gprat_cu_multiserver_create.argtypes = [_ip, ctypes.c_int, _i64, ctypes.c_int, ctypes.POINTER(_vp)]
    lib.gprat_cu_multiserver_destroy.argtypes = [_vp]
    lib.gprat_cu_multiserver_add_model.argtypes = lib.gprat_cu_server_add_model.argtypes
    lib.gprat_cu_multiserver_submit_predict.argtypes = lib.gprat_cu_server_submit_predict.argtypes
    lib.gprat_cu_multiserver_submit_fit.argtypes = lib.gprat_cu_server_submit_fit.argtypes
    lib.gprat_cu_multiserver_wait.argtypes = lib.gprat_cu_server_wait.argtypes
    lib.gprat_cu_multiserver_stats.argtypes = lib.gprat_cu_server_stats.argtypes
    lib.gprat_cu_multiserver_replica_completed.argtypes = [_vp, ctypes.c_int, _i64p]
    lib.gprat_cu_multiserver_set_replication.argtypes = [_vp, ctypes.c_int]
    lib.gprat_cu_multiserver_resident_bytes.argtypes = [_vp, ctypes.c_int, _i64p]
    lib.gprat_cu_test_multiserver_fail_copy.argtypes = [_vp, ctypes.c_int]
    return lib


lib = _load()


def declared_symbols() -> List[str]:
    """Every function name declared in include/gprat_cu.h."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(gprat_cu_[a-z_0-9]+)\s*\(", text)))


def check(rc: int) -> None:
    if rc == OK:
        return
    msg = lib.gprat_cu_last_error().decode()
    if rc == ERR_NOT_SPD:
        raise NotPositiveDefiniteError(rc, msg)
    raise GpratCudaError(rc, msg)


def device_count() -> int:
    c = ctypes.c_int(0)
    check(lib.gprat_cu_device_count(ctypes.byref(c)))
    return c.value


def stats_reset() -> None:
    check(lib.gprat_cu_stats_reset())


def stats_enable_timing(enable: bool) -> None:
    check(lib.gprat_cu_stats_enable_timing(int(bool(enable))))


def stats_read() -> dict:
    """{'launches', 'gemm_launches', 'gemm_ms', 'gemm_flops'} since the last reset."""
    a, b = ctypes.c_int64(), ctypes.c_int64()
    c, d = ctypes.c_double(), ctypes.c_double()
    check(lib.gprat_cu_stats_read(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d)))
    return {"launches": a.value, "gemm_launches": b.value, "gemm_ms": c.value, "gemm_flops": d.value}


def steps_enable(enable: bool) -> None:
    check(lib.gprat_cu_steps_enable(int(bool(enable))))


def steps_reset() -> None:
    check(lib.gprat_cu_steps_reset())


def steps_csv() -> str:
    """Per-phase step timers as CSV text: label,calls,total_ms,mean_ms."""
    need = ctypes.c_int64()
    check(lib.gprat_cu_steps_csv(None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(int(need.value) + 64)
    check(lib.gprat_cu_steps_csv(buf, len(buf), ctypes.byref(need)))
    return buf.value.decode()


def steps() -> dict:
    """{label: (calls, total_ms)} from steps_csv()."""
    out = {}
    for line in steps_csv().strip().splitlines()[1:]:
        label, calls, total, _ = line.rsplit(",", 3)
        out[label] = (int(calls), float(total))
    return out


def test_tc_gemm(kind: int, A: np.ndarray, B: np.ndarray, C: np.ndarray, alpha: float, beta: float,
                 lower: bool = False, rowsq: Optional[np.ndarray] = None, tile_mode: int = 0) -> None:
    """Runs the tcgen05 GEMM C = beta*C + alpha*A B^T in place on float32 arrays
    (kind 0 = TF32, 1 = BF16; tile_mode 0 = automatic, 1 = 128x128, 2 = 128x256,
    3 = 256x256 on a CTA pair)."""
    _fp = ctypes.POINTER(ctypes.c_float)
    for a in (A, B, C):
        if a.dtype != np.float32 or not a.flags.c_contiguous:
            raise ValueError("A, B and C must be C-contiguous float32 arrays")
    M, K = A.shape
    N = B.shape[0]
    rp = rowsq.ctypes.data_as(_dp) if rowsq is not None else None
    check(lib.gprat_cu_test_tc_gemm(int(kind), M, N, K, A.ctypes.data_as(_fp), K, B.ctypes.data_as(_fp), K,
                                    C.ctypes.data_as(_fp), C.shape[1], float(alpha), float(beta), int(bool(lower)),
                                    rp, int(tile_mode)))


def test_trsv(kind: int, L: np.ndarray, b: np.ndarray, max_ctas: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """Runs the fused triangular solves on the lower triangle of L (n x n):
    returns (L^-1 b, L^-T b).  kind 0 = FP64 factor, 1 = FP32 factor and
    inverses (the mixed path's preconditioner)."""
    L = np.ascontiguousarray(L, dtype=np.float64)
    b = _arr(b)
    n = L.shape[0]
    xf, xb = np.empty(n), np.empty(n)
    check(lib.gprat_cu_test_trsv(int(kind), n, _p(L), _p(b), _p(xf), _p(xb), int(max_ctas)))
    return xf, xb


def test_set_wait_budget(polls: int) -> None:
    """Poll budget of the fused triangular solves' waits on the current device
    (negative: the default).  Tests use 0 to make a wait give up."""
    check(lib.gprat_cu_test_set_wait_budget(int(polls)))


def test_oz_split(src: np.ndarray, s: int, block: bool) -> Tuple[np.ndarray, np.ndarray]:
    """Splits src (rows x cols, cols a multiple of 128) into s int8 digit
    planes on the device; returns (digits[s, rows, cols], exponents) with one
    exponent per row and 128-column block (block=False) or per 128 x 128 block."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    rows, cols = src.shape
    digits = np.empty((s, rows, cols), dtype=np.int8)
    er = (rows + 127) // 128 if block else rows
    exps = np.empty((er, cols // 128), dtype=np.int32)
    check(lib.gprat_cu_test_oz_split(rows, cols, _p(src), int(s), int(bool(block)),
                                     digits.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)),
                                     exps.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
    return digits, exps


def test_oz_gemm(A: np.ndarray, B: np.ndarray, C: np.ndarray, alpha: float, beta: float, s: int, groups: int = 0,
                 lower: bool = False, rowsq: Optional[np.ndarray] = None, max_ctas: int = 0) -> None:
    """Runs the int8-emulated FP64 GEMM C = beta*C + alpha*A B^T in place
    (A: M x K, B: N x K, C: M x N, float64, K a multiple of 128; s digit
    planes, `groups` digit groups kept, 0 = s)."""
    for a in (A, B, C):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("A, B and C must be C-contiguous float64 arrays")
    M, K = A.shape
    N = B.shape[0]
    rp = _p(rowsq) if rowsq is not None else None
    check(lib.gprat_cu_test_oz_gemm(M, N, K, _p(A), _p(B), _p(C), float(alpha), float(beta), int(bool(lower)),
                                    int(s), int(groups), rp, int(max_ctas)))


def _arr(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _hyper(h) -> np.ndarray:
    h = _arr(h)
    if h.size != 3:
        raise ValueError("hyper-parameters must be (lengthscale, vertical_lengthscale, noise_variance)")
    return h


class CudaGP:
    """One device-resident GP (handle over gprat_cu_gp)."""

    def __init__(self, x: Sequence[float], y: Sequence[float], n_tiles: int, n_tile_size: int, n_reg: int = 8,
                 device: int = 0):
        self.x, self.y = _arr(x), _arr(y)
        self.n_tiles, self.n_tile_size, self.n_reg = int(n_tiles), int(n_tile_size), int(n_reg)
        self.n = self.n_tiles * self.n_tile_size
        h = ctypes.c_void_p()
        check(lib.gprat_cu_gp_create(int(device), _p(self.x), self.x.size, _p(self.y), self.y.size, self.n_tiles,
                                     self.n_tile_size, self.n_reg, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.gprat_cu_gp_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def set_precision(self, precision: int) -> None:
        check(lib.gprat_cu_gp_set_precision(self._h, int(precision)))

    def set_int8_slices(self, slices: int) -> None:
        """Digit planes of the int8-emulated FP64 products (PREC_FP64_INT8), 3..7."""
        check(lib.gprat_cu_gp_set_int8_slices(self._h, int(slices)))

    def set_int8_groups(self, factor_groups: int, variance_groups: int) -> None:
        """Digit groups kept in the factorisation's trailing updates and the
        variance solve's updates (int8-emulated products; 0 = all of them)."""
        check(lib.gprat_cu_gp_set_int8_groups(self._h, int(factor_groups), int(variance_groups)))

    def cholesky(self, hyper) -> List[Optional[np.ndarray]]:
        nt, t = self.n_tiles, self.n_tile_size
        out = np.empty(nt * nt * t * t)
        check(lib.gprat_cu_cholesky(self._h, _p(_hyper(hyper)), _p(out)))
        tiles = out.reshape(nt * nt, t * t)
        return [tiles[i * nt + j].copy() if j <= i else None for i in range(nt) for j in range(nt)]

    def predict(self, hyper, xt, m_tiles: int, m_tile_size: int) -> np.ndarray:
        xt = _arr(xt)
        mean = np.empty(max(m_tiles * m_tile_size, 1))
        check(lib.gprat_cu_predict(self._h, _p(_hyper(hyper)), _p(xt), xt.size, m_tiles, m_tile_size, _p(mean)))
        return mean[: m_tiles * m_tile_size]

    def predict_with_uncertainty(self, hyper, xt, m_tiles: int, m_tile_size: int) -> Tuple[np.ndarray, np.ndarray]:
        xt = _arr(xt)
        m = m_tiles * m_tile_size
        mean, var = np.empty(max(m, 1)), np.empty(max(m, 1))
        check(lib.gprat_cu_predict_with_uncertainty(self._h, _p(_hyper(hyper)), _p(xt), xt.size, m_tiles,
                                                    m_tile_size, _p(mean), _p(var)))
        return mean[:m], var[:m]

    def predict_with_full_cov(self, hyper, xt, m_tiles: int, m_tile_size: int) -> Tuple[np.ndarray, np.ndarray]:
        xt = _arr(xt)
        m = m_tiles * m_tile_size
        mean, var = np.empty(max(m, 1)), np.empty(max(m, 1))
        check(lib.gprat_cu_predict_with_full_cov(self._h, _p(_hyper(hyper)), _p(xt), xt.size, m_tiles, m_tile_size,
                                                 _p(mean), _p(var)))
        return mean[:m], var[:m]

    def predict_full_covariance(self, hyper, xt, m: int) -> Tuple[np.ndarray, np.ndarray]:
        xt = _arr(xt)
        mean, cov = np.empty(max(m, 1)), np.empty(max(m * m, 1))
        check(lib.gprat_cu_predict_full_covariance(self._h, _p(_hyper(hyper)), _p(xt), xt.size, m, _p(mean),
                                                   _p(cov)))
        return mean[:m], cov[: m * m].reshape(m, m)

    def compute_loss(self, hyper) -> float:
        v = ctypes.c_double()
        check(lib.gprat_cu_compute_loss(self._h, _p(_hyper(hyper)), ctypes.byref(v)))
        return v.value

    def loss_grad(self, hyper) -> Tuple[float, np.ndarray]:
        v = ctypes.c_double()
        g = np.empty(3)
        check(lib.gprat_cu_loss_grad(self._h, _p(_hyper(hyper)), ctypes.byref(v), _p(g)))
        return v.value, g

    def optimize_step(self, params, adam, trainable, iter_: int) -> Tuple[float, np.ndarray]:
        p = _arr(params).copy()
        a = _arr(adam)
        t = np.ascontiguousarray([int(bool(v)) for v in trainable], dtype=np.int32)
        v = ctypes.c_double()
        check(lib.gprat_cu_optimize_step(self._h, _p(p), _p(a), t.ctypes.data_as(_ip), int(iter_), ctypes.byref(v)))
        return v.value, p

    def optimize(self, params, adam, trainable, opt_iter: int) -> Tuple[np.ndarray, np.ndarray]:
        p = _arr(params).copy()
        a = _arr(adam)
        t = np.ascontiguousarray([int(bool(v)) for v in trainable], dtype=np.int32)
        losses = np.empty(max(int(opt_iter), 1))
        check(lib.gprat_cu_optimize(self._h, _p(p), _p(a), t.ctypes.data_as(_ip), int(opt_iter), _p(losses)))
        return losses[: int(opt_iter)], p

    def fit_predict_device(self, hyper, d_xt: int, n_xt: int, m: int, d_mean: int, d_var: Optional[int],
                           stream: int = 0) -> None:
        check(lib.gprat_cu_fit_predict_device(self._h, _p(_hyper(hyper)), ctypes.c_void_p(d_xt), n_xt, m,
                                              ctypes.c_void_p(d_mean), ctypes.c_void_p(d_var or 0),
                                              ctypes.c_void_p(stream)))

    def check_status(self) -> None:
        check(lib.gprat_cu_check_status(self._h))

    def pcg_iterations(self) -> int:
        v = ctypes.c_int()
        check(lib.gprat_cu_gp_pcg_iterations(self._h, ctypes.byref(v)))
        return v.value
