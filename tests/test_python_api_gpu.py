"""The reference's own integration test (test/src/output_correctness.cpp:58-309)
replayed through the drop-in Python API: `import gprat_b200 as gprat`,
data loaded with GP_data from files, results compared with the golden
output.json at the test's tolerance (WithinRel 1e6*DBL_EPSILON)."""
import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu

REL = 1e6 * np.finfo(float).eps


def rel_err(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


@pytest.fixture(scope="module")
def gprat():
    import gprat_b200 as g
    assert g.gpu_count() >= 1
    return g


@pytest.fixture()
def data_files(tmp_path, known_answer):
    paths = {}
    for name in ("training_input", "training_output", "test_input"):
        p = tmp_path / f"{name}.txt"
        p.write_text("\n".join(repr(v) for v in known_answer["raw"][name]) + "\n")
        paths[name] = str(p)
    return paths


@pytest.mark.parametrize("use_gpu_ctor", [False, True])
def test_reference_integration_test(gprat, known_answer, data_files, use_gpu_ctor):
    n_train = n_test = 128
    n_tiles, n_reg = 4, 8
    tile_size = gprat.compute_train_tile_size(n_train, n_tiles)
    m_tiles, m_tile_size = gprat.compute_test_tiles(n_test, n_tiles, tile_size)
    train_in = gprat.GP_data(data_files["training_input"], n_train, n_reg)
    train_out = gprat.GP_data(data_files["training_output"], n_train, n_reg)
    test_in = gprat.GP_data(data_files["test_input"], n_test, n_reg)
    args = (train_in.data, train_out.data, n_tiles, tile_size, n_reg, [1.0, 1.0, 0.1], [True, True, True])
    gp = gprat.GP(*args, gpu_id=0, n_streams=1) if use_gpu_ctor else gprat.GP(*args)
    gprat.start_hpx([], 2)
    exp = known_answer["expected"]
    tiles = gp.cholesky()
    for got, want in zip(tiles, exp["choleksy"]):
        assert len(got) == len(want)
        if want:
            assert rel_err(got, want) <= REL
    mean, var = gp.predict_with_uncertainty(test_in.data, m_tiles, m_tile_size)
    assert rel_err(mean, exp["sum"][0]) <= REL and rel_err(var, exp["sum"][1]) <= REL
    mean, var = gp.predict_with_full_cov(test_in.data, m_tiles, m_tile_size)
    assert rel_err(mean, exp["full"][0]) <= REL and rel_err(var, exp["full"][1]) <= REL
    assert rel_err(gp.predict(test_in.data, m_tiles, m_tile_size), exp["pred"]) <= REL
    losses = gp.optimize(gprat.AdamParams(0.1, 0.9, 0.999, 1e-8, 3))
    assert rel_err(losses, exp["losses"]) <= REL
    gprat.stop_hpx()


def test_optimize_step_updates_kernel_params(gprat, ref_cases):
    n, d, T = (int(v) for v in ref_cases["opt_cfg"])
    x, y, _ = O.synthetic(n, 16, d)
    gp = gprat.GP(list(x), list(y), n // T, T, d, [0.5, 2.0, 0.5], [True, True, True])
    adam = gprat.AdamParams(0.1, 0.9, 0.999, 1e-8)
    for it in range(5):
        loss = gp.optimize_step(adam, it)
        assert rel_err(loss, ref_cases["opt_losses"][it]) < 1e-10
        kp = gp.kernel_params
        got = [kp.lengthscale, kp.vertical_lengthscale, kp.noise_variance] + list(kp.m_T) + list(kp.w_T)
        assert rel_err(got, ref_cases["opt_params"][it]) < 1e-10


def test_untrainable_parameters_stay_fixed(gprat):
    x, y, _ = O.synthetic(256, 16, 8)
    gp = gprat.GP(list(x), list(y), 2, 128, 8, [0.7, 1.3, 0.2], [True, False, True])
    gp.optimize(gprat.AdamParams(0.1, opt_iter=2))
    assert gp.kernel_params.vertical_lengthscale == 1.3
    assert gp.kernel_params.lengthscale != 0.7 and gp.kernel_params.noise_variance != 0.2


def test_calculate_loss_and_gradient(gprat):
    n, d, T = 512, 8, 128
    x, y, _ = O.synthetic(n, 16, d)
    gp = gprat.GP(list(x), list(y), n // T, T, d, [0.9, 1.1, 0.07], [True, True, True])
    o = O.OracleGP(x, y, n // T, T, d, (0.9, 1.1, 0.07))
    loss, g = o.gradient()
    assert rel_err(gp.compute_loss(), loss) < 1e-10
    lg = gp.loss_and_gradient()
    assert rel_err(lg[0], loss) < 1e-10 and rel_err(lg[1:], g) < 1e-10


def test_full_covariance_extension(gprat):
    n, m, d, T = 256, 40, 8, 64
    x, y, xt = O.synthetic(n, m, d)
    gp = gprat.GP(list(x), list(y), n // T, T, d)
    mean, cov = gp.predict_full_covariance(list(xt), m)
    want = O.OracleGP(x, y, n // T, T, d, (1.0, 1.0, 0.1)).posterior_covariance(xt, m)
    assert np.max(np.abs(np.array(cov).reshape(m, m) - want)) < 1e-10


def test_invalid_test_input_raises_value_error(gprat):
    x, y, _ = O.synthetic(256, 16, 8)
    gp = gprat.GP(list(x), list(y), 2, 128, 8)
    with pytest.raises(ValueError, match="test input"):
        gp.predict([0.0] * 4, 1, 8)
