"""Test infrastructure: ctypes binding of the reference's own CPU GP path.

``oracle/_ref/libgprat_ref.so`` is the reference's CPU sources compiled
unmodified (recipe: ``oracle/Makefile``; C layer: ``oracle/ref_capi.cpp``).
Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, as the checker.  The product never imports it.

``RefGP`` mirrors ``gprat::GP`` (core/include/gprat_c.hpp:54-228).
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libgprat_ref.so")

_lib = None
_started = False

_dp = ctypes.POINTER(ctypes.c_double)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise FileNotFoundError(f"compiled reference not built: {LIB_PATH} (run make -C oracle)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.gprat_ref_last_error.restype = ctypes.c_char_p
    lib.gprat_ref_create.restype = ctypes.c_void_p
    lib.gprat_ref_create.argtypes = [
        _dp, ctypes.c_long, _dp, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
    ]
    lib.gprat_ref_destroy.argtypes = [ctypes.c_void_p]
    lib.gprat_ref_start.argtypes = [ctypes.c_int]
    lib.gprat_ref_get_params.argtypes = [ctypes.c_void_p, _dp]
    lib.gprat_ref_set_params.argtypes = [ctypes.c_void_p, _dp]
    lib.gprat_ref_cholesky.argtypes = [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_ubyte)]
    lib.gprat_ref_predict.argtypes = [ctypes.c_void_p, _dp, ctypes.c_long, ctypes.c_int, ctypes.c_int, _dp]
    for name in ("gprat_ref_predict_with_uncertainty", "gprat_ref_predict_with_full_cov"):
        getattr(lib, name).argtypes = [ctypes.c_void_p, _dp, ctypes.c_long, ctypes.c_int, ctypes.c_int, _dp, _dp]
    lib.gprat_ref_calculate_loss.argtypes = [ctypes.c_void_p, _dp]
    lib.gprat_ref_optimize.argtypes = [
        ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp]
    lib.gprat_ref_optimize_step.argtypes = [
        ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
        ctypes.c_int, _dp]
    lib.gprat_ref_compute_test_tiles.argtypes = [
        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    _lib = lib
    return lib


def start(n_threads: Optional[int] = None) -> None:
    """Starts the reference's task runtime (HPX: ``--hpx:threads=N``)."""
    global _started
    lib = _load()
    if _started:
        return
    if n_threads is None:
        n_threads = os.cpu_count() or 1
    _check(lib.gprat_ref_start(int(n_threads)))
    _started = True


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(_load().gprat_ref_last_error().decode())


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def compute_test_tiles(n_test: int, n_tiles: int, n_tile_size: int) -> Tuple[int, int]:
    lib = _load()
    a, b = ctypes.c_int(), ctypes.c_int()
    _check(lib.gprat_ref_compute_test_tiles(n_test, n_tiles, n_tile_size, ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


class RefGP:
    """The reference's gprat::GP on the CPU (task runtime + OpenBLAS)."""

    def __init__(self, x: Sequence[float], y: Sequence[float], n_tiles: int, n_tile_size: int, n_reg: int = 8,
                 kernel_params: Sequence[float] = (1.0, 1.0, 0.1), trainable: Sequence[bool] = (True, True, True)):
        lib = _load()
        start()
        self._x = np.ascontiguousarray(x, dtype=np.float64)
        self._y = np.ascontiguousarray(y, dtype=np.float64)
        self.n_tiles, self.n_tile_size, self.n_reg = int(n_tiles), int(n_tile_size), int(n_reg)
        h = lib.gprat_ref_create(_ptr(self._x), self._x.size, _ptr(self._y), self._y.size, self.n_tiles,
                                 self.n_tile_size, self.n_reg, float(kernel_params[0]), float(kernel_params[1]),
                                 float(kernel_params[2]), int(trainable[0]), int(trainable[1]), int(trainable[2]))
        if not h:
            raise RuntimeError(lib.gprat_ref_last_error().decode())
        self._h = ctypes.c_void_p(h)

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.gprat_ref_destroy(self._h)
            self._h = None

    # params: (lengthscale, vertical_lengthscale, noise_variance), m_T[3], w_T[3]
    def get_params(self) -> np.ndarray:
        out = np.zeros(9)
        _check(_lib.gprat_ref_get_params(self._h, _ptr(out)))
        return out

    def set_params(self, params: Sequence[float]) -> None:
        p = np.ascontiguousarray(params, dtype=np.float64)
        _check(_lib.gprat_ref_set_params(self._h, _ptr(p)))

    def cholesky(self) -> List[Optional[np.ndarray]]:
        nt, t = self.n_tiles, self.n_tile_size
        out = np.zeros(nt * nt * t * t)
        present = np.zeros(nt * nt, dtype=np.uint8)
        _check(_lib.gprat_ref_cholesky(self._h, _ptr(out), present.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))))
        tiles = out.reshape(nt * nt, t * t)
        return [tiles[k].copy() if present[k] else None for k in range(nt * nt)]

    def predict(self, xt, m_tiles: int, m_tile_size: int) -> np.ndarray:
        xt = np.ascontiguousarray(xt, dtype=np.float64)
        mean = np.zeros(m_tiles * m_tile_size)
        _check(_lib.gprat_ref_predict(self._h, _ptr(xt), xt.size, m_tiles, m_tile_size, _ptr(mean)))
        return mean

    def predict_with_uncertainty(self, xt, m_tiles: int, m_tile_size: int):
        xt = np.ascontiguousarray(xt, dtype=np.float64)
        mean, var = np.zeros(m_tiles * m_tile_size), np.zeros(m_tiles * m_tile_size)
        _check(_lib.gprat_ref_predict_with_uncertainty(self._h, _ptr(xt), xt.size, m_tiles, m_tile_size, _ptr(mean),
                                                       _ptr(var)))
        return mean, var

    def predict_with_full_cov(self, xt, m_tiles: int, m_tile_size: int):
        xt = np.ascontiguousarray(xt, dtype=np.float64)
        mean, var = np.zeros(m_tiles * m_tile_size), np.zeros(m_tiles * m_tile_size)
        _check(_lib.gprat_ref_predict_with_full_cov(self._h, _ptr(xt), xt.size, m_tiles, m_tile_size, _ptr(mean),
                                                    _ptr(var)))
        return mean, var

    def calculate_loss(self) -> float:
        v = ctypes.c_double()
        _check(_lib.gprat_ref_calculate_loss(self._h, ctypes.byref(v)))
        return v.value

    def optimize(self, lr=0.001, b1=0.9, b2=0.999, eps=1e-8, opt_iter=0) -> np.ndarray:
        out = np.zeros(max(int(opt_iter), 1))
        _check(_lib.gprat_ref_optimize(self._h, lr, b1, b2, eps, int(opt_iter), _ptr(out)))
        return out[: int(opt_iter)]

    def optimize_step(self, iter_: int, lr=0.001, b1=0.9, b2=0.999, eps=1e-8, opt_iter=0) -> float:
        v = ctypes.c_double()
        _check(_lib.gprat_ref_optimize_step(self._h, lr, b1, b2, eps, int(opt_iter), int(iter_), ctypes.byref(v)))
        return v.value

    def gradient(self, lr=0.001, b1=0.9, b2=0.999, eps=1e-8) -> np.ndarray:
        """Gradient of the reference's loss w.r.t. the unconstrained
        hyper-parameters at the current point, recovered from the first Adam
        moment (core/src/cpu/tiled_algorithms.cpp:422-432:
        m_new = b1*m_old + (1-b1)*g).  The model's parameters and moments are
        restored afterwards."""
        saved = self.get_params()
        self.optimize_step(0, lr, b1, b2, eps)
        after = self.get_params()
        self.set_params(saved)
        return (after[3:6] - b1 * saved[3:6]) / (1.0 - b1)
