"""Host-side semantics of the drop-in Python API (module `gprat` of the
reference, bindings/gprat_py.cpp and bindings/utils_py.cpp) that need no GPU."""
import os

import numpy as np
import pytest

import gprat_b200 as gprat


def test_tile_helpers_match_reference_semantics():
    # core/src/utils_c.cpp:8-52
    assert gprat.compute_train_tiles(1024, 64) == 16
    assert gprat.compute_train_tile_size(128, 4) == 32
    assert gprat.compute_train_tile_size(130, 4) == 32  # floors
    assert gprat.compute_test_tiles(128, 4, 32) == (4, 32)
    assert gprat.compute_test_tiles(200, 4, 64) == (4, 50)  # truncates
    with pytest.raises(RuntimeError):
        gprat.compute_train_tiles(10, 0)
    with pytest.raises(RuntimeError):
        gprat.compute_train_tile_size(10, 0)


def test_gp_data_prefixes_zeros(tmp_path):
    # GP_data(path, n, n_reg) -> n_reg - 1 zeros then n values (core/src/gprat_c.cpp:15-21)
    p = tmp_path / "d.txt"
    p.write_text("\n".join(str(v) for v in [0.5, -1.25, 2.0, 3.5]) + "\n")
    d = gprat.GP_data(str(p), 3, 4)
    assert d.n_samples == 3 and d.n_regressors == 4 and d.file_path == str(p)
    assert d.data == [0.0, 0.0, 0.0, 0.5, -1.25, 2.0]


def test_gp_data_errors(tmp_path):
    with pytest.raises(RuntimeError, match="File not found"):
        gprat.GP_data(str(tmp_path / "missing.txt"), 3, 8)
    p = tmp_path / "short.txt"
    p.write_text("1.0\n2.0\n")
    with pytest.raises(RuntimeError, match="Expected 5"):
        gprat.GP_data(str(p), 5, 1)


def test_adam_params_defaults_and_fields():
    a = gprat.AdamParams()
    assert (a.learning_rate, a.beta1, a.beta2, a.epsilon, a.opt_iter) == (0.001, 0.9, 0.999, 1e-8, 0)
    a.learning_rate = 0.1
    a.opt_iter = 3
    assert "learning_rate=0.10000000" in repr(a) and "opt_iter=3" in repr(a)


def test_gp_construction_and_repr():
    x = list(np.linspace(0, 1, 20))
    y = list(np.linspace(1, 2, 16))
    gp = gprat.GP(x, y, 4, 4, 5, [1.5, 0.5, 0.01], [True, False, True])
    r = repr(gp)
    assert r.startswith("Kernel_Params: [lengthscale=1.500000000000, vertical_lengthscale=0.500000000000")
    assert "trainable_params v=0" in r and "Target: [CPU]" in r and r.endswith("n_tiles=4, n_tile_size=4")
    assert gp.get_input_data() == x and gp.get_output_data() == y
    assert gp.n_reg == 5
    kp = gp.kernel_params
    assert (kp.lengthscale, kp.vertical_lengthscale, kp.noise_variance) == (1.5, 0.5, 0.01)
    assert kp.m_T == [0.0, 0.0, 0.0] and kp.w_T == [0.0, 0.0, 0.0]
    kp.lengthscale = 2.0
    gp.kernel_params = kp
    assert gp.kernel_params.lengthscale == 2.0


def test_runtime_helpers_are_harmless():
    gprat.start_hpx([], 2)
    gprat.suspend_hpx()
    gprat.resume_hpx()
    gprat.stop_hpx()
    assert gprat.compiled_with_cuda() is True
    assert gprat.gpu_count() >= 0


@pytest.mark.skipif(gprat.gpu_count() > 0, reason="checks the no-device error path")
def test_no_device_errors_are_runtime_errors():
    with pytest.raises(RuntimeError, match="not available"):
        gprat.GP([0.0] * 20, [0.0] * 16, 4, 4, 5, gpu_id=0)
    gp = gprat.GP([0.0] * 20, [0.0] * 16, 4, 4, 5)
    with pytest.raises(RuntimeError):
        gp.compute_loss()
