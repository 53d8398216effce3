"""Parity at the benchmark configurations' full sizes against the reference's
own CPU code (compiled from source; fixtures in tests/golden/ref_large.npz,
made by tests/golden/make_golden.py --large):

  C1: n_train 16384, n_test 4096, d 8, 32 x 32 tiles of 512, (1.0, 1.0, 0.1)
  C2: n_train 32768, n_test 8192, d 64, 32 x 32 tiles of 1024, (4.0, 1.0, 0.01)

FP64 path: mean, variance and loss within 1e-10 relative of the reference;
Cholesky tiles through their sums of squares (1e-10), plus three 32 x 32
corners per element at the reference test's own bar, WithinRel with
eps = 1e6 * DBL_EPSILON = 2.2e-10 (test/src/output_correctness.cpp:209-216):
at n = 16384 the per-element relative deviation of the smallest entries of
L is about 1.4e-10.  The int8-emulated FP64 path: mean and variance within
1e-8.
"""
import os

import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "ref_large.npz")
FP64_TOL = 1e-10
ELEMENT_TOL = 1e6 * np.finfo(np.float64).eps  # the reference test's WithinRel bar
INT8_TOL = 1e-8


@pytest.fixture(scope="module")
def large():
    if not os.path.exists(FIXTURE):
        pytest.fail("tests/golden/ref_large.npz is missing (tests/golden/make_golden.py --large)")
    return dict(np.load(FIXTURE))


@pytest.fixture(scope="module")
def capi():
    from gprat_b200 import capi as c

    assert c.device_count() >= 1
    return c


def case(large, tag):
    if f"{tag}_cfg" not in large:
        pytest.fail(f"fixture {tag} missing from ref_large.npz")
    n, m, d, T, mt, mts = (int(v) for v in large[f"{tag}_cfg"])
    x, y, xt = O.synthetic(n, m, d)
    return dict(n=n, m=m, d=d, T=T, mt=mt, mts=mts, x=x, y=y, xt=xt, h=tuple(large[f"{tag}_hyper"]))


def mean_err(got, want):
    """Largest deviation relative to the largest predicted mean (means cross zero)."""
    return float(np.max(np.abs(got - want)) / np.max(np.abs(want)))


def var_err(got, want):
    """Largest per-point relative deviation of the variance."""
    return float(np.max(np.abs(got - want) / np.abs(want)))


@pytest.mark.parametrize("tag", ["c1", "c2"])
def test_fp64_predict_and_loss(capi, large, tag):
    c = case(large, tag)
    gp = capi.CudaGP(c["x"], c["y"], c["n"] // c["T"], c["T"], c["d"])
    mean, var = gp.predict_with_uncertainty(c["h"], c["xt"], c["mt"], c["mts"])
    loss = gp.compute_loss(c["h"])
    em, ev = mean_err(mean, large[f"{tag}_mean"]), var_err(var, large[f"{tag}_var"])
    el = abs(loss - large[f"{tag}_loss"][0]) / abs(large[f"{tag}_loss"][0])
    pm = float(np.max(np.abs(mean - large[f"{tag}_mean"]) / np.abs(large[f"{tag}_mean"])))
    print(f"{tag} FP64: mean {em:.2e} (per point {pm:.2e}), var {ev:.2e}, loss {el:.2e}")
    assert em <= FP64_TOL
    assert ev <= FP64_TOL
    assert el <= FP64_TOL
    gp.close()


@pytest.mark.parametrize("tag", ["c1", "c2"])
def test_fp64_cholesky_tiles(capi, large, tag):
    c = case(large, tag)
    nt, T = c["n"] // c["T"], c["T"]
    gp = capi.CudaGP(c["x"], c["y"], nt, T, c["d"])
    tiles = gp.cholesky(c["h"])
    gp.close()
    sumsq = np.array([np.dot(t, t) if t is not None else 0.0 for t in tiles])
    want = large[f"{tag}_tile_sumsq"]
    present = want > 0
    assert np.array_equal(present, np.array([t is not None for t in tiles]))
    esq = float(np.max(np.abs(sumsq[present] - want[present]) / want[present]))
    corners = [
        (tiles[0].reshape(T, T)[:32, :32], large[f"{tag}_corner_00"]),
        (tiles[nt * nt - 1].reshape(T, T)[-32:, -32:], large[f"{tag}_corner_last"]),
        (tiles[(nt - 1) * nt].reshape(T, T)[:32, :32], large[f"{tag}_corner_low"]),
    ]
    # WithinRel: |a - b| <= eps * max(|a|, |b|), per element
    ec = max(float(np.max(np.abs(g - w) / np.maximum(np.maximum(np.abs(w), np.abs(g)), 1e-300)))
             for g, w in corners)
    print(f"{tag} FP64 cholesky: tile sums of squares {esq:.2e}, corners {ec:.2e}")
    assert esq <= FP64_TOL
    assert ec <= ELEMENT_TOL


@pytest.mark.parametrize("tag,slices", [("c1", 5), ("c2", 5), ("c2", 6)])
def test_int8_fp64_predict(capi, large, tag, slices):
    c = case(large, tag)
    gp = capi.CudaGP(c["x"], c["y"], c["n"] // c["T"], c["T"], c["d"])
    gp.set_precision(capi.PREC_FP64_INT8)
    gp.set_int8_slices(slices)
    mean, var = gp.predict_with_uncertainty(c["h"], c["xt"], c["mt"], c["mts"])
    loss = gp.compute_loss(c["h"])
    em, ev = mean_err(mean, large[f"{tag}_mean"]), var_err(var, large[f"{tag}_var"])
    el = abs(loss - large[f"{tag}_loss"][0]) / abs(large[f"{tag}_loss"][0])
    print(f"{tag} int8 s={slices}: mean {em:.2e}, var {ev:.2e}, loss {el:.2e}")
    assert em <= INT8_TOL
    assert ev <= INT8_TOL
    gp.close()
