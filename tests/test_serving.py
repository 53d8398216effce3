"""Serving layer (gprat_cu_server_*): resident models, continuous batching of
uneven predict requests, fits running beside them, admission by memory.

The property under test: every predict result is bit-identical to the same
request run alone, whatever else shares its batch or the device, and equals
the FP64 oracle (FP64 servers) to 1e-10 relative.
"""
import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def serving():
    from gprat_b200 import capi, serving as S
    assert capi.device_count() >= 1
    return capi, S


def _models(d=8):
    specs = [(1024, 128, (1.0, 1.0, 0.1)), (2048, 256, (0.8, 1.2, 0.05)), (1536, 128, (1.3, 0.9, 0.2))]
    out = []
    for i, (n, T, h) in enumerate(specs):
        x, y, _ = O.synthetic(n, 16, d, seeds=(10 + i, 20 + i, 30 + i))
        out.append(dict(n=n, T=T, h=h, x=x, y=y, d=d))
    return out


def _requests(n_models, d, count, seed=5):
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(count):
        mid = int(rng.integers(0, n_models))
        m = int(np.exp(rng.uniform(0, np.log(700))))
        series = rng.uniform(-1.0, 1.0, size=m + d - 1)
        reqs.append((mid, m, series))
    return reqs


@pytest.mark.parametrize("prec", [0, 1, 3])  # FP64, mixed TF32, int8-emulated FP64
def test_mixed_batches_bit_identical_to_alone(serving, prec):
    capi, S = serving
    models = _models()
    reqs = _requests(len(models), 8, 40)
    with S.Server(precision=prec) as sv:
        ids = [sv.add_model(md["x"], md["y"], md["n"] // md["T"], md["T"], md["d"], md["h"]) for md in models]
        # alone: one request in the server at a time
        alone = []
        for mid, m, series in reqs:
            rid = sv.submit_predict(ids[mid], series, m)
            mean, var, got_mid, lat = sv.wait(rid)
            assert got_mid == ids[mid] and lat >= 0.0
            alone.append((mean, var))
        b0 = sv.stats().batches
        # mix: all requests in flight together, plus a fit on the side
        fx, fy, _ = O.synthetic(1024, 16, 8, seeds=(7, 8, 9))
        fit_id = sv.submit_fit(fx, fy, 8, 128, 8, (1.1, 1.0, 0.1))
        rids = [sv.submit_predict(ids[mid], series, m) for mid, m, series in reqs]
        mixed = [sv.wait(r) for r in rids]
        _, _, new_mid, _ = sv.wait(fit_id)
        st = sv.stats()
        assert st.batches - b0 < len(reqs), "requests of one model were never batched together"
        for (mean_a, var_a), (mean_b, var_b, _, _) in zip(alone, mixed):
            assert np.array_equal(mean_a, mean_b)
            assert np.array_equal(var_a, var_b)
        # the fitted model serves like the others
        series = np.random.default_rng(3).uniform(-1, 1, 100 + 7)
        mean, var, _, _ = sv.wait(sv.submit_predict(new_mid, series, 100))
        o = O.OracleGP(fx, fy, 8, 128, 8, (1.1, 1.0, 0.1))
        om, ov = o.predict_with_uncertainty(series, 1, 100)
        tol_m, tol_v = {0: (1e-10, 1e-10), 1: (1e-8, 1.5e-2), 3: (1e-8, 1e-8)}[prec]
        assert np.max(np.abs(mean - om)) / np.max(np.abs(om)) <= tol_m
        assert np.max(np.abs(var - ov) / ov) <= tol_v
        assert st.completed >= 2 * len(reqs)
        assert 0.0 < st.p50_ms <= st.p99_ms


def test_results_match_oracle_fp64(serving):
    capi, S = serving
    models = _models()
    reqs = _requests(len(models), 8, 12, seed=11)
    with S.Server(precision=capi.PREC_FP64) as sv:
        ids = [sv.add_model(md["x"], md["y"], md["n"] // md["T"], md["T"], md["d"], md["h"]) for md in models]
        rids = [sv.submit_predict(ids[mid], series, m) for mid, m, series in reqs]
        res = [sv.wait(r) for r in rids]
    oracles = [O.OracleGP(md["x"], md["y"], md["n"] // md["T"], md["T"], md["d"], md["h"]) for md in models]
    for (mid, m, series), (mean, var, _, _) in zip(reqs, res):
        om, ov = oracles[mid].predict_with_uncertainty(series, 1, m)
        assert np.max(np.abs(mean - om)) <= 1e-10 * max(1.0, np.max(np.abs(om)))
        assert np.max(np.abs(var - ov) / ov) <= 1e-10


def test_admission_rejects_fit_over_budget(serving):
    capi, S = serving
    with S.Server(memory_budget_bytes=64 << 20) as sv:
        x, y, _ = O.synthetic(4096, 16, 8)
        rid = sv.submit_fit(x, y, 16, 256, 8, (1.0, 1.0, 0.1))
        with pytest.raises(capi.GpratCudaError) as e:
            sv.wait(rid)
        assert e.value.code == capi.ERR_OOM
        # the server keeps serving what fits
        x, y, _ = O.synthetic(512, 16, 8)
        mid = sv.add_model(x, y, 4, 128, 8, (1.0, 1.0, 0.1))
        mean, var, _, _ = sv.wait(sv.submit_predict(mid, np.linspace(-1, 1, 40), 33))
        assert mean.shape == (33,) and np.all(var > 0)


def test_invalid_requests(serving):
    capi, S = serving
    with S.Server() as sv:
        with pytest.raises(capi.GpratCudaError):
            sv.submit_predict(0, np.zeros(10), 3)  # no model yet
        x, y, _ = O.synthetic(512, 16, 8)
        mid = sv.add_model(x, y, 4, 128, 8, (1.0, 1.0, 0.1))
        with pytest.raises(capi.GpratCudaError):
            sv.submit_predict(mid, np.zeros(5), 3)  # series shorter than m + d - 1
        with pytest.raises(capi.GpratCudaError):
            sv.wait(12345)  # unknown request
