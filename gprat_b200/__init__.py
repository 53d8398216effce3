"""gprat_b200 — GPRat's GP-regression hot path on NVIDIA B200 (sm_100a).

``import gprat_b200 as gprat`` gives the reference's Python API (module
``gprat``: GP, GP_data, AdamParams, compute_test_tiles, ...), implemented by
the pybind11 module ``gprat_b200.gprat`` over the C++ mirror of
``gprat::GP`` (libgprat.so) and the CUDA kernels behind the C ABI in
include/gprat_cu.h (libgprat_cuda.so).  The native libraries are built
in-tree by ``python -m gprat_b200.build``.  Attributes load the native
module on first use; without a build that fails loudly -- there is no CPU
fallback.
"""
import importlib as _importlib

_native = None


def _load_native():
    global _native
    if _native is None:
        try:
            _native = _importlib.import_module(".gprat", __name__)
        except ImportError as e:
            raise ImportError("gprat_b200 native module is not built; run `python -m gprat_b200.build`: "
                              f"{e}") from e
    return _native


_SUBMODULES = {"build", "capi", "autograd", "serving", "gprat"}


def __getattr__(name):
    if name in _SUBMODULES:
        return _importlib.import_module("." + name, __name__)
    if name.startswith("__"):
        raise AttributeError(name)
    return getattr(_load_native(), name)


def __dir__():
    return sorted(set(globals()) | {n for n in dir(_load_native()) if not n.startswith("_")})
