"""The oracle is pinned before anything is compared against it.

1. The numpy restatement (oracle/gprat_oracle.py) reproduces the reference's
   own known-answer file (data/data_1024/output.json) at the reference test's
   tolerance (test/src/output_correctness.cpp:209-247: WithinRel 1e6*DBL_EPSILON).
2. The reference's CPU code compiled from source (oracle/_ref) reproduces it too.
3. The numpy restatement matches golden vectors produced by the compiled
   reference on seeded synthetic inputs (tests/golden/ref_cases.npz).
"""
import numpy as np
import pytest

from oracle import gprat_oracle as O
from oracle import ref

REL = 1e6 * np.finfo(float).eps  # the reference test's WithinRel tolerance


def rel_err(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def check_known_answer(gp_cls, g, opt):
    n_tiles = g["n_tiles"]
    T = g["n_train"] // n_tiles
    mt, mts = O.compute_test_tiles(g["n_test"], n_tiles, T)
    gp = gp_cls(g["train_in"], g["train_out"], n_tiles, T, g["n_reg"], g["kernel_params"])
    exp = g["expected"]
    tiles = gp.cholesky()
    assert len(tiles) == len(exp["choleksy"])
    for got, want in zip(tiles, exp["choleksy"]):
        if len(want) == 0:
            assert got is None
        else:
            assert rel_err(got, want) <= REL
    mean, var = gp.predict_with_uncertainty(g["test_in"], mt, mts)
    assert rel_err(mean, exp["sum"][0]) <= REL and rel_err(var, exp["sum"][1]) <= REL
    mean, var = gp.predict_with_full_cov(g["test_in"], mt, mts)
    assert rel_err(mean, exp["full"][0]) <= REL and rel_err(var, exp["full"][1]) <= REL
    assert rel_err(gp.predict(g["test_in"], mt, mts), exp["pred"]) <= REL
    assert rel_err(opt(gp), exp["losses"]) <= REL


def test_numpy_oracle_known_answer(known_answer):
    lr, b1, b2, eps, it = known_answer["adam"]
    check_known_answer(O.OracleGP, known_answer, lambda gp: gp.optimize(O.Adam(lr, b1, b2, eps, int(it))))


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built (make -C oracle)")
def test_compiled_reference_known_answer(known_answer):
    lr, b1, b2, eps, it = known_answer["adam"]
    check_known_answer(ref.RefGP, known_answer, lambda gp: gp.optimize(lr, b1, b2, eps, int(it)))


@pytest.mark.parametrize("tag", ["c0", "ragged", "d64"])
def test_numpy_oracle_matches_reference_vectors(ref_cases, tag):
    n, m, d, T, mt, mts = (int(v) for v in ref_cases[f"{tag}_cfg"])
    x, y, xt = O.synthetic(n, m, d)
    gp = O.OracleGP(x, y, n // T, T, d, ref_cases[f"{tag}_hyper"])
    mean, var = gp.predict_with_uncertainty(xt, mt, mts)
    assert rel_err(mean, ref_cases[f"{tag}_mean"]) < 1e-9
    assert rel_err(var, ref_cases[f"{tag}_var"]) < 1e-9
    fm, fv = gp.predict_with_full_cov(xt, mt, mts)
    assert rel_err(fv, ref_cases[f"{tag}_full_var"]) < 1e-9
    assert rel_err(gp.predict(xt, mt, mts), ref_cases[f"{tag}_pred"]) < 1e-9
    assert rel_err(gp.calculate_loss(), ref_cases[f"{tag}_loss"][0]) < 1e-12
    tiles = gp.cholesky()
    sums = np.array([t.sum() if t is not None else np.nan for t in tiles])
    want = ref_cases[f"{tag}_tile_sums"]
    assert np.array_equal(np.isnan(sums), np.isnan(want))
    ok = ~np.isnan(want)
    assert np.allclose(sums[ok], want[ok], rtol=1e-9, atol=1e-9)


def test_numpy_oracle_matches_reference_optimizer(ref_cases):
    n, d, T = (int(v) for v in ref_cases["opt_cfg"])
    x, y, _ = O.synthetic(n, 16, d)
    gp = O.OracleGP(x, y, n // T, T, d, (0.5, 2.0, 0.5))
    adam = O.Adam(0.1, 0.9, 0.999, 1e-8)
    for it in range(5):
        _, g = gp.gradient()
        assert rel_err(g, ref_cases["opt_grads"][it]) < 1e-9
        loss = gp.optimize_step(adam, it)
        assert rel_err(loss, ref_cases["opt_losses"][it]) < 1e-12
        got = np.array(gp.hyper + gp.m_T + gp.w_T)
        assert rel_err(got, ref_cases["opt_params"][it]) < 1e-9


def test_compute_test_tiles_semantics():
    # utils::compute_test_tiles (core/src/utils_c.cpp:34-52): divisible -> same tile size,
    # otherwise same number of tiles with a truncating tile size.
    assert O.compute_test_tiles(128, 4, 32) == (4, 32)
    assert O.compute_test_tiles(200, 4, 64) == (4, 50)
    assert O.compute_test_tiles(10, 4, 64) == (4, 2)
    assert O.compute_test_tiles(4096, 32, 512) == (8, 512)


def test_synthetic_generator_is_seeded():
    a = O.synthetic(64, 32, 8)
    b = O.synthetic(64, 32, 8)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    x, y, xt = a
    assert x.size == 64 + 8 and xt.size == 32 + 8 and y.size == 64
