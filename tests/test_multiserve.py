"""Replica serving (gprat_cu_multiserver_*): every model replicated on each
replica (fitted once and copied, or fitted on every replica), predict
requests spread over the replicas by outstanding test points.

The property under test: a result is bit-identical to the same request on a
single server, whichever replica served it, and the replicas share the load.
The replicas here are two servers on device 0 (one GPU is visible); the
routing and the per-replica state are the same for distinct devices.
"""
import numpy as np
import pytest

from oracle import gprat_oracle as O

pytestmark = pytest.mark.gpu

BUDGET = 4 << 30


@pytest.fixture(scope="module")
def serving():
    from gprat_b200 import capi, serving as S
    assert capi.device_count() >= 1
    return capi, S


def _models(d=8):
    specs = [(1024, 128, (1.0, 1.0, 0.1)), (2048, 256, (0.8, 1.2, 0.05))]
    out = []
    for i, (n, T, h) in enumerate(specs):
        x, y, _ = O.synthetic(n, 16, d, seeds=(40 + i, 50 + i, 60 + i))
        out.append(dict(n=n, T=T, h=h, x=x, y=y, d=d))
    return out


def _requests(n_models, d, count, seed=9):
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(count):
        mid = int(rng.integers(0, n_models))
        m = int(np.exp(rng.uniform(0, np.log(500))))
        reqs.append((mid, m, rng.uniform(-1.0, 1.0, size=m + d - 1)))
    return reqs


def _add(sv, models):
    return [sv.add_model(md["x"], md["y"], md["n"] // md["T"], md["T"], md["d"], md["h"]) for md in models]


@pytest.mark.parametrize("prec,replication", [(0, 0), (1, 0), (1, 1)])
def test_replicas_bit_identical_to_single_server(serving, prec, replication):
    capi, S = serving
    models = _models()
    reqs = _requests(len(models), 8, 30)
    with S.Server(memory_budget_bytes=BUDGET, precision=prec) as sv:
        ids = _add(sv, models)
        single = [sv.wait(sv.submit_predict(ids[mid], series, m)) for mid, m, series in reqs]
    with S.MultiServer([0, 0], memory_budget_bytes=BUDGET, precision=prec, replication=replication) as ms:
        gids = _add(ms, models)
        assert gids == [0, 1]
        rids = [ms.submit_predict(gids[mid], series, m) for mid, m, series in reqs]
        multi = [ms.wait(r) for r in rids]
        per_replica = ms.replica_completed()
        st = ms.stats()
    for (mid, _, _), (mean_a, var_a, _, _), (mean_b, var_b, got_mid, lat) in zip(reqs, single, multi):
        assert got_mid == gids[mid] and lat >= 0.0
        assert np.array_equal(mean_a, mean_b)
        assert np.array_equal(var_a, var_b)
    assert sum(per_replica) == len(reqs)
    assert min(per_replica) > 0, f"one replica served nothing: {per_replica}"
    assert st.completed == len(reqs) and 0.0 < st.p50_ms <= st.p99_ms


@pytest.mark.parametrize("prec,replication", [(0, 0), (0, 1), (2, 0)])
def test_fit_replicated_on_every_replica(serving, prec, replication):
    capi, S = serving
    fx, fy, _ = O.synthetic(1024, 16, 8, seeds=(71, 72, 73))
    hyper = (1.1, 1.0, 0.1)
    series = np.random.default_rng(4).uniform(-1, 1, 200 + 7)
    with S.Server(memory_budget_bytes=BUDGET, precision=prec) as sv:
        _, _, mid, _ = sv.wait(sv.submit_fit(fx, fy, 8, 128, 8, hyper))
        ref_mean, ref_var, _, _ = sv.wait(sv.submit_predict(mid, series, 200))
    with S.MultiServer([0, 0], memory_budget_bytes=BUDGET, precision=prec, replication=replication) as ms:
        _, _, gid, _ = ms.wait(ms.submit_fit(fx, fy, 8, 128, 8, hyper))
        # enough requests that both replicas serve the fitted model
        rids = [ms.submit_predict(gid, series, 200) for _ in range(6)]
        res = [ms.wait(r) for r in rids]
        assert min(ms.replica_completed()) > 0
    for mean, var, got, _ in res:
        assert got == gid
        assert np.array_equal(mean, ref_mean) and np.array_equal(var, ref_var)
    o = O.OracleGP(fx, fy, 8, 128, 8, hyper)
    om, ov = o.predict_with_uncertainty(series, 1, 200)
    tol_m, tol_v = {0: (1e-10, 1e-10), 1: (1e-8, 1.5e-2), 2: (1e-8, 5e-2)}[prec]
    assert np.max(np.abs(ref_mean - om)) <= tol_m * max(1.0, np.max(np.abs(om)))
    assert np.max(np.abs(ref_var - ov) / ov) <= tol_v


def test_multiserver_invalid_requests(serving):
    capi, S = serving
    with pytest.raises(capi.GpratCudaError):
        S.MultiServer([])
    with pytest.raises(capi.GpratCudaError):
        S.MultiServer([0, 10_000])  # no such device; the first replica is released
    with pytest.raises(capi.GpratCudaError):
        S.MultiServer([0], replication=7)
    with S.MultiServer([0, 0], memory_budget_bytes=BUDGET) as ms:
        with pytest.raises(capi.GpratCudaError):
            ms.submit_predict(0, np.zeros(10), 3)  # no model yet
        x, y, _ = O.synthetic(512, 16, 8)
        mid = ms.add_model(x, y, 4, 128, 8, (1.0, 1.0, 0.1))
        with pytest.raises(capi.GpratCudaError):
            ms.submit_predict(mid, np.zeros(5), 3)  # series shorter than m + d - 1
        with pytest.raises(capi.GpratCudaError):
            ms.wait(12345)
        # still serving after the rejected requests
        mean, var, _, _ = ms.wait(ms.submit_predict(mid, np.linspace(-1, 1, 40), 33))
        assert mean.shape == (33,) and np.all(var > 0)
        assert ms.replica_completed() in ([1, 0], [0, 1])


def test_failed_copy_frees_every_replica(serving):
    """A replicated fit whose copy to one replica fails (an error made on the
    host by the test hook) fails the request and leaves nothing resident
    without a global id: the fitted original on the first replica is freed
    too.  The same holds for a synchronous add.  The server keeps serving, and
    its results match the oracle."""
    capi, S = serving
    fx, fy, _ = O.synthetic(1024, 16, 8, seeds=(81, 82, 83))
    hyper = (1.0, 1.0, 0.1)
    series = np.random.default_rng(8).uniform(-1, 1, 50 + 7)
    with S.MultiServer([0, 0], memory_budget_bytes=BUDGET, precision=capi.PREC_FP64,
                       replication=capi.REPLICATE_COPY) as ms:
        before = ms.resident_bytes()
        ms.fail_next_copy(1)
        with pytest.raises(capi.GpratCudaError) as err:
            ms.wait(ms.submit_fit(fx, fy, 8, 128, 8, hyper))
        assert err.value.code == capi.ERR_OOM
        assert ms.resident_bytes() == before
        ms.fail_next_copy(1)
        with pytest.raises(capi.GpratCudaError):
            ms.add_model(fx, fy, 8, 128, 8, hyper)
        assert ms.resident_bytes() == before
        _, _, gid, _ = ms.wait(ms.submit_fit(fx, fy, 8, 128, 8, hyper))
        assert all(b > a for a, b in zip(before, ms.resident_bytes()))
        # submitted together, so the outstanding-points routing spreads them over both replicas
        tickets = [ms.submit_predict(gid, series, 50) for _ in range(4)]
        results = [ms.wait(t) for t in tickets]
        assert min(ms.replica_completed()) > 0
    om, ov = O.OracleGP(fx, fy, 8, 128, 8, hyper).predict_with_uncertainty(series, 1, 50)
    for mean, var, got, _ in results:
        assert got == gid
        assert np.max(np.abs(mean - om)) <= 1e-10 * max(1.0, np.max(np.abs(om)))
        assert np.max(np.abs(var - ov) / ov) <= 1e-10
