// Replica serving over several GPUs: one resident-model server per device
// (serve.cu), every model replicated on each, predict requests sent to the
// replica with the fewest test points outstanding.  Test points are
// independent given a model's factor and alpha, so this scales predict
// throughput with the number of GPUs with no change to the algorithm.  A
// model is fitted once, on the first replica, and its fitted state (factor,
// alpha, training data) is copied to the others over NVLink (peer copies,
// copy engines only), or, in the refit mode, fitted on every replica at once
// (the pipeline is deterministic, so the copies are identical either way).
// No counterpart in the reference.
#include "gp_state.cuh"

#include <algorithm>
#include <chrono>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace gprat_cu
{
void set_last_error(const std::string &message);
int server_add_model_copy(gprat_cu_server *dst, gprat_cu_server *src, int src_model, const double *train_in,
                          int64_t n_in, const double *train_out, int64_t n_out, int n_tiles, int n_tile_size,
                          int n_regressors, int *model_id);
int server_release_model(gprat_cu_server *sv, int model_id);
int64_t server_resident_bytes(gprat_cu_server *sv);
}

using namespace gprat_cu;

namespace
{

struct Pending
{
    bool fit = false;
    int replica = -1;                // predict: the replica that serves it
    int64_t rows = 0;                // predict: test points (load accounting)
    int model = -1;                  // predict: the global model id
    std::vector<int64_t> local_ids;  // per replica (fit) or one (predict)
    // fit in the copy mode: the training data and tiling for the copies
    std::vector<double> x, y;
    int n_tiles = 0, T = 0, d = 0;
};

}  // namespace

struct gprat_cu_multiserver
{
    std::vector<int> devices;
    std::vector<gprat_cu_server *> servers;
    std::mutex mtx;
    std::vector<int64_t> outstanding;          // test points submitted and not yet waited, per replica
    std::vector<int64_t> completed;            // requests waited, per replica
    std::vector<std::vector<int>> model_ids;   // global model id -> the replicas' model ids
    std::unordered_map<int64_t, Pending> pending;
    std::vector<double> latencies_ms;
    int64_t next_id = 1;
    int replication = GPRAT_CU_REPLICATE_COPY;
    int fail_copy_replica = -1;  // test hook: the next copy to this replica reports a failure
};

namespace
{

template <typename F>
int guarded_ms(F &&f)
{
    try
    {
        f();
        set_last_error("");
        return GPRAT_CU_OK;
    }
    catch (const Error &e)
    {
        set_last_error(e.what());
        return e.code;
    }
    catch (const std::bad_alloc &)
    {
        set_last_error("host out of memory");
        return GPRAT_CU_ERR_OOM;
    }
    catch (const std::exception &e)
    {
        set_last_error(e.what());
        return GPRAT_CU_ERR_INVALID_ARG;
    }
}

void check_rc(int rc)
{
    if (rc != GPRAT_CU_OK)
    {
        throw Error(rc, gprat_cu_last_error());
    }
}

void require_ms(bool c, const char *msg)
{
    if (!c)
    {
        throw Error(GPRAT_CU_ERR_INVALID_ARG, msg);
    }
}

// Runs f(replica) on every replica at once; the first failure is rethrown.
template <typename F>
void on_every_replica(gprat_cu_multiserver *ms, F &&f)
{
    const int n = static_cast<int>(ms->servers.size());
    std::vector<int> rc(n, GPRAT_CU_OK);
    std::vector<std::string> msg(n);
    std::vector<std::thread> th;
    for (int r = 0; r < n; ++r)
    {
        th.emplace_back(
            [&, r]
            {
                rc[r] = f(r);
                if (rc[r] != GPRAT_CU_OK)
                {
                    msg[r] = gprat_cu_last_error();
                }
            });
    }
    for (auto &t : th)
    {
        t.join();
    }
    for (int r = 0; r < n; ++r)
    {
        if (rc[r] != GPRAT_CU_OK)
        {
            throw Error(rc[r], "replica " + std::to_string(r) + ": " + msg[r]);
        }
    }
}

// Copies replica 0's model id0 to every other replica; ids[0] = id0.
void copy_to_replicas(gprat_cu_multiserver *ms, int id0, const double *x, int64_t nx, const double *y, int64_t ny,
                      int n_tiles, int T, int d, std::vector<int> &ids)
{
    ids.assign(ms->servers.size(), -1);
    ids[0] = id0;
    int fail = -1;
    {
        std::lock_guard<std::mutex> lk(ms->mtx);
        std::swap(fail, ms->fail_copy_replica);
    }
    on_every_replica(ms,
                     [&](int r)
                     {
                         if (r == 0)
                         {
                             return static_cast<int>(GPRAT_CU_OK);
                         }
                         if (r == fail)
                         {
                             set_last_error("copy to the replica failed (injected by the test hook)");
                             return static_cast<int>(GPRAT_CU_ERR_OOM);
                         }
                         return server_add_model_copy(ms->servers[r], ms->servers[0], id0, x, nx, y, ny, n_tiles, T,
                                                      d, &ids[r]);
                     });
}

// A replicated fit that failed somewhere: the replicas' models that did
// come into being (ids[r] >= 0) are freed, so no unreachable copy stays
// resident.
void release_replicas(gprat_cu_multiserver *ms, const std::vector<int> &ids)
{
    for (size_t r = 0; r < ids.size() && r < ms->servers.size(); ++r)
    {
        if (ids[r] >= 0)
        {
            server_release_model(ms->servers[r], ids[r]);
        }
    }
}

// Lets each replica's device read every other replica's memory directly
// (NVLink), where the devices differ and support it.
void enable_peer_access(const std::vector<int> &devices)
{
    int prev = 0;
    cudaGetDevice(&prev);
    for (int a : devices)
    {
        for (int b : devices)
        {
            int can = 0;
            if (a == b || cudaDeviceCanAccessPeer(&can, a, b) != cudaSuccess || !can)
            {
                continue;
            }
            cudaSetDevice(a);
            const cudaError_t e = cudaDeviceEnablePeerAccess(b, 0);
            if (e == cudaErrorPeerAccessAlreadyEnabled)
            {
                cudaGetLastError();
            }
            else
            {
                GPRAT_CUDA_CHECK(e);
            }
        }
    }
    cudaSetDevice(prev);
}

}  // namespace

extern "C" {

int gprat_cu_multiserver_create(const int *devices, int n_devices, int64_t memory_budget_bytes, int precision,
                                gprat_cu_multiserver **out)
{
    return guarded_ms(
        [&]
        {
            require_ms(out != nullptr && devices != nullptr, "arguments must not be NULL");
            require_ms(n_devices >= 1, "a multi-server needs at least one device");
            *out = nullptr;
            auto ms = std::make_unique<gprat_cu_multiserver>();
            for (int r = 0; r < n_devices; ++r)
            {
                gprat_cu_server *sv = nullptr;
                const int rc = gprat_cu_server_create(devices[r], memory_budget_bytes, precision, &sv);
                if (rc != GPRAT_CU_OK)
                {
                    const std::string m = gprat_cu_last_error();
                    for (gprat_cu_server *s : ms->servers)
                    {
                        gprat_cu_server_destroy(s);
                    }
                    throw Error(rc, m);
                }
                ms->servers.push_back(sv);
                ms->devices.push_back(devices[r]);
            }
            ms->outstanding.assign(n_devices, 0);
            ms->completed.assign(n_devices, 0);
            try
            {
                enable_peer_access(ms->devices);
            }
            catch (...)
            {
                for (gprat_cu_server *sv : ms->servers)
                {
                    gprat_cu_server_destroy(sv);
                }
                throw;
            }
            *out = ms.release();
        });
}

int gprat_cu_multiserver_destroy(gprat_cu_multiserver *ms)
{
    return guarded_ms(
        [&]
        {
            if (ms == nullptr)
            {
                return;
            }
            for (gprat_cu_server *s : ms->servers)
            {
                gprat_cu_server_destroy(s);
            }
            delete ms;
        });
}

int gprat_cu_multiserver_add_model(gprat_cu_multiserver *ms, const double *train_in, int64_t n_in,
                                   const double *train_out, int64_t n_out, int n_tiles, int n_tile_size,
                                   int n_regressors, const double hyper[3], int *model_id)
{
    return guarded_ms(
        [&]
        {
            require_ms(ms != nullptr && model_id != nullptr, "arguments must not be NULL");
            std::vector<int> ids(ms->servers.size(), -1);
            try
            {
                if (ms->replication == GPRAT_CU_REPLICATE_COPY)
                {
                    check_rc(gprat_cu_server_add_model(ms->servers[0], train_in, n_in, train_out, n_out, n_tiles,
                                                       n_tile_size, n_regressors, hyper, &ids[0]));
                    copy_to_replicas(ms, ids[0], train_in, n_in, train_out, n_out, n_tiles, n_tile_size,
                                     n_regressors, ids);
                }
                else
                {
                    on_every_replica(ms,
                                     [&](int r)
                                     {
                                         return gprat_cu_server_add_model(ms->servers[r], train_in, n_in, train_out,
                                                                          n_out, n_tiles, n_tile_size, n_regressors,
                                                                          hyper, &ids[r]);
                                     });
                }
            }
            catch (...)
            {
                release_replicas(ms, ids);  // no replica keeps a model that has no global id
                throw;
            }
            std::lock_guard<std::mutex> lk(ms->mtx);
            ms->model_ids.push_back(ids);
            *model_id = static_cast<int>(ms->model_ids.size()) - 1;
        });
}

int gprat_cu_multiserver_submit_predict(gprat_cu_multiserver *ms, int model_id, const double *test_in,
                                        int64_t n_test_in, int m, int64_t *request_id)
{
    return guarded_ms(
        [&]
        {
            require_ms(ms != nullptr && request_id != nullptr, "arguments must not be NULL");
            int replica = 0;
            int local_model = -1;
            {
                std::lock_guard<std::mutex> lk(ms->mtx);
                require_ms(model_id >= 0 && model_id < static_cast<int>(ms->model_ids.size()), "unknown model id");
                for (int r = 1; r < static_cast<int>(ms->servers.size()); ++r)
                {
                    if (ms->outstanding[r] < ms->outstanding[replica])
                    {
                        replica = r;
                    }
                }
                local_model = ms->model_ids[model_id][replica];
                ms->outstanding[replica] += m;  // reserved before the submit, released if it fails
            }
            int64_t local = 0;
            const int rc = gprat_cu_server_submit_predict(ms->servers[replica], local_model, test_in, n_test_in, m,
                                                          &local);
            std::lock_guard<std::mutex> lk(ms->mtx);
            if (rc != GPRAT_CU_OK)
            {
                ms->outstanding[replica] -= m;
                check_rc(rc);
            }
            Pending p;
            p.replica = replica;
            p.rows = m;
            p.model = model_id;
            p.local_ids = { local };
            const int64_t id = ms->next_id++;
            ms->pending.emplace(id, std::move(p));
            *request_id = id;
        });
}

int gprat_cu_multiserver_submit_fit(gprat_cu_multiserver *ms, const double *train_in, int64_t n_in,
                                    const double *train_out, int64_t n_out, int n_tiles, int n_tile_size,
                                    int n_regressors, const double hyper[3], int64_t *request_id)
{
    return guarded_ms(
        [&]
        {
            require_ms(ms != nullptr && request_id != nullptr, "arguments must not be NULL");
            Pending p;
            p.fit = true;
            const bool copy = ms->replication == GPRAT_CU_REPLICATE_COPY;
            if (copy)
            {
                require_ms(train_in != nullptr && train_out != nullptr && n_in >= 0 && n_out >= 0,
                           "arguments must not be NULL");
                p.x.assign(train_in, train_in + n_in);
                p.y.assign(train_out, train_out + n_out);
                p.n_tiles = n_tiles;
                p.T = n_tile_size;
                p.d = n_regressors;
            }
            p.local_ids.assign(copy ? 1 : ms->servers.size(), 0);
            for (size_t r = 0; r < p.local_ids.size(); ++r)
            {
                const int rc = gprat_cu_server_submit_fit(ms->servers[r], train_in, n_in, train_out, n_out, n_tiles,
                                                          n_tile_size, n_regressors, hyper, &p.local_ids[r]);
                if (rc != GPRAT_CU_OK)
                {
                    // the replicas that accepted the fit finish it; their models are freed
                    const std::string m = gprat_cu_last_error();
                    std::vector<int> done(r, -1);
                    for (size_t q = 0; q < r; ++q)
                    {
                        gprat_cu_server_wait(ms->servers[q], p.local_ids[q], nullptr, nullptr, &done[q], nullptr);
                    }
                    release_replicas(ms, done);
                    throw Error(rc, "replica " + std::to_string(r) + ": " + m);
                }
            }
            std::lock_guard<std::mutex> lk(ms->mtx);
            const int64_t id = ms->next_id++;
            ms->pending.emplace(id, std::move(p));
            *request_id = id;
        });
}

int gprat_cu_multiserver_wait(gprat_cu_multiserver *ms, int64_t request_id, double *mean, double *var,
                              int *model_id, double *latency_ms)
{
    return guarded_ms(
        [&]
        {
            require_ms(ms != nullptr, "multi-server must not be NULL");
            Pending p;
            {
                std::lock_guard<std::mutex> lk(ms->mtx);
                auto it = ms->pending.find(request_id);
                require_ms(it != ms->pending.end(), "unknown or already completed request id");
                p = std::move(it->second);
                ms->pending.erase(it);
            }
            if (!p.fit)
            {
                double lat = 0.0;
                const int rc = gprat_cu_server_wait(ms->servers[p.replica], p.local_ids[0], mean, var, nullptr, &lat);
                std::lock_guard<std::mutex> lk(ms->mtx);
                ms->outstanding[p.replica] -= p.rows;
                check_rc(rc);
                ms->completed[p.replica] += 1;
                ms->latencies_ms.push_back(lat);
                if (latency_ms != nullptr)
                {
                    *latency_ms = lat;
                }
                if (model_id != nullptr)
                {
                    *model_id = p.model;
                }
                return;
            }
            // a fit: every replica's copy, then one global model id
            std::vector<int> ids(ms->servers.size(), -1);
            double worst = 0.0;
            if (p.local_ids.size() == 1)
            {
                // fitted on replica 0; the copies to the others count in the latency
                check_rc(gprat_cu_server_wait(ms->servers[0], p.local_ids[0], nullptr, nullptr, &ids[0], &worst));
                const auto t0 = std::chrono::steady_clock::now();
                try
                {
                    copy_to_replicas(ms, ids[0], p.x.data(), static_cast<int64_t>(p.x.size()), p.y.data(),
                                     static_cast<int64_t>(p.y.size()), p.n_tiles, p.T, p.d, ids);
                }
                catch (...)
                {
                    release_replicas(ms, ids);  // the original on replica 0 and the copies that succeeded
                    throw;
                }
                worst += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            }
            else
            {
                std::vector<double> lats(ms->servers.size(), 0.0);
                try
                {
                    on_every_replica(ms,
                                     [&](int r)
                                     {
                                         return gprat_cu_server_wait(ms->servers[r], p.local_ids[r], nullptr, nullptr,
                                                                     &ids[r], &lats[r]);
                                     });
                }
                catch (...)
                {
                    release_replicas(ms, ids);  // the replicas whose fit succeeded
                    throw;
                }
                for (double l : lats)
                {
                    worst = std::max(worst, l);
                }
            }
            std::lock_guard<std::mutex> lk(ms->mtx);
            ms->model_ids.push_back(ids);
            if (model_id != nullptr)
            {
                *model_id = static_cast<int>(ms->model_ids.size()) - 1;
            }
            if (latency_ms != nullptr)
            {
                *latency_ms = worst;
            }
        });
}

int gprat_cu_multiserver_stats(gprat_cu_multiserver *ms, double *p50_ms, double *p99_ms, double *predictions_per_s,
                               int64_t *completed, int64_t *batches)
{
    return guarded_ms(
        [&]
        {
            require_ms(ms != nullptr, "multi-server must not be NULL");
            double pps = 0.0;
            int64_t nb = 0;
            for (gprat_cu_server *s : ms->servers)
            {
                double a = 0, b = 0, c = 0;
                int64_t d = 0, e = 0;
                check_rc(gprat_cu_server_stats(s, &a, &b, &c, &d, &e));
                pps += c;
                nb += e;
            }
            std::lock_guard<std::mutex> lk(ms->mtx);
            std::vector<double> l = ms->latencies_ms;
            std::sort(l.begin(), l.end());
            auto pct = [&](double q)
            {
                if (l.empty())
                {
                    return 0.0;
                }
                const double pos = q * static_cast<double>(l.size() - 1);
                const size_t lo = static_cast<size_t>(pos);
                const size_t hi = std::min(lo + 1, l.size() - 1);
                return l[lo] + (pos - static_cast<double>(lo)) * (l[hi] - l[lo]);
            };
            if (p50_ms != nullptr)
            {
                *p50_ms = pct(0.50);
            }
            if (p99_ms != nullptr)
            {
                *p99_ms = pct(0.99);
            }
            if (predictions_per_s != nullptr)
            {
                *predictions_per_s = pps;
            }
            if (completed != nullptr)
            {
                int64_t c = 0;
                for (int64_t v : ms->completed)
                {
                    c += v;
                }
                *completed = c;
            }
            if (batches != nullptr)
            {
                *batches = nb;
            }
        });
}

int gprat_cu_multiserver_set_replication(gprat_cu_multiserver *ms, int mode)
{
    return guarded_ms(
        [&]
        {
            require_ms(ms != nullptr, "multi-server must not be NULL");
            require_ms(mode == GPRAT_CU_REPLICATE_COPY || mode == GPRAT_CU_REPLICATE_REFIT,
                       "replication mode must be GPRAT_CU_REPLICATE_COPY or GPRAT_CU_REPLICATE_REFIT");
            std::lock_guard<std::mutex> lk(ms->mtx);
            ms->replication = mode;
        });
}

int gprat_cu_multiserver_resident_bytes(gprat_cu_multiserver *ms, int replica, int64_t *bytes)
{
    return guarded_ms(
        [&]
        {
            require_ms(ms != nullptr && bytes != nullptr, "arguments must not be NULL");
            require_ms(replica >= 0 && replica < static_cast<int>(ms->servers.size()), "unknown replica");
            *bytes = server_resident_bytes(ms->servers[replica]);
        });
}

int gprat_cu_test_multiserver_fail_copy(gprat_cu_multiserver *ms, int replica)
{
    return guarded_ms(
        [&]
        {
            require_ms(ms != nullptr, "multi-server must not be NULL");
            require_ms(replica >= 1 && replica < static_cast<int>(ms->servers.size()),
                       "the injected failure needs a replica other than the first");
            std::lock_guard<std::mutex> lk(ms->mtx);
            ms->fail_copy_replica = replica;
        });
}

int gprat_cu_multiserver_replica_completed(gprat_cu_multiserver *ms, int replica, int64_t *completed)
{
    return guarded_ms(
        [&]
        {
            require_ms(ms != nullptr && completed != nullptr, "arguments must not be NULL");
            std::lock_guard<std::mutex> lk(ms->mtx);
            require_ms(replica >= 0 && replica < static_cast<int>(ms->servers.size()), "unknown replica");
            *completed = ms->completed[replica];
        });
}

}  // extern "C"
