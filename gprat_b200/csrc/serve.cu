// Serving loop: fitted GP models resident in HBM, asynchronous predict and
// fit requests, continuous batching, admission by memory, latency statistics.
// No counterpart in the reference (every reference call refactorises K and
// copies everything back to the host).
//
// Threads:
//   scheduler : forms batches and launches them.  Pending predict requests
//               of one model are concatenated into one batch (each request
//               keeps its own test series; a per-row offset table tells the
//               cross-covariance kernel where each row's window starts) and
//               run as one launch sequence on that model's stream: assembly,
//               fused mean, variance solve.  Each model has one batch in
//               flight; batches of different models run concurrently on their
//               own streams.  Requests that arrive while a batch runs join the
//               next batch as soon as the model's slot and the memory budget
//               allow.
//   fitter    : fit requests (a new model) run on their own streams, so they
//               overlap with predict batches on the device.
// Memory: every model reserves its factor, weights and the working set of a
// batch of RESERVED_ROWS test points when it is created, so steady-state
// batches allocate nothing (an allocation or free would synchronise the
// device and stall every other stream).  A batch beyond the reservation (a
// single request larger than RESERVED_ROWS) is charged its extra working set
// while it runs.  Resident models plus those extras stay below the budget; a
// batch takes requests in arrival order while they fit.
#include "gp_state.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace gprat_cu
{
void set_last_error(const std::string &message);
}

using namespace gprat_cu;
using Clock = std::chrono::steady_clock;

namespace
{

constexpr int MAX_BATCH_ROWS = 8192;  // rows per batch unless one request alone is larger
constexpr int RESERVED_ROWS = MAX_BATCH_ROWS;

struct Request
{
    int64_t id = 0;
    bool fit = false;
    int model = -1;
    int m = 0;
    std::vector<double> series;
    // fit inputs
    std::vector<double> x, y;
    int n_tiles = 0, T = 0, d = 0;
    double hyper[3] = { 0, 0, 0 };
    // results
    std::vector<double> mean, var;
    int new_model = -1;
    int status = GPRAT_CU_OK;
    std::string error;
    bool done = false;
    Clock::time_point t_submit, t_done;
};

struct PinnedBuf
{
    void *p = nullptr;
    size_t cap = 0;
    void ensure(size_t bytes)
    {
        if (bytes <= cap)
        {
            return;
        }
        if (p != nullptr)
        {
            cudaFreeHost(p);
        }
        p = nullptr;
        cap = 0;
        GPRAT_CUDA_CHECK(cudaMallocHost(&p, bytes));
        cap = bytes;
    }
    ~PinnedBuf()
    {
        if (p != nullptr)
        {
            cudaFreeHost(p);
        }
    }
};

struct Model
{
    gprat_cu_gp *gp = nullptr;
    int d = 0;
    int64_t resident = 0;
    // batch buffers
    DevBuf<double> d_series, d_mean, d_var;
    DevBuf<int64_t> d_offsets;
    PinnedBuf h_in, h_out;
    cudaEvent_t done_ev = nullptr;
    bool busy = false;
    bool released = false;  // device state freed (server_release_model); the id stays unused
    std::vector<Request *> inflight;
    int64_t inflight_bytes = 0;
    ~Model()
    {
        if (done_ev != nullptr)
        {
            cudaEventDestroy(done_ev);
        }
        if (gp != nullptr)
        {
            gprat_cu_gp_destroy(gp);
        }
    }
};

}  // namespace

// Most device memory a server reserves in the allocation pool when it starts
// (at most its budget).
constexpr int64_t POOL_RESERVE_MAX = int64_t{ 64 } << 30;

struct gprat_cu_server
{
    int device = 0;
    int precision = GPRAT_CU_PREC_FP64;
    int64_t budget = 0;
    int64_t pool_reserved = 0;  // bytes pool_hold keeps for this server
    int64_t used = 0;
    std::mutex mtx;
    std::condition_variable cv_work, cv_done, cv_fit;
    std::deque<Request *> pending;      // predict requests, arrival order
    std::deque<Request *> pending_fit;  // fit requests
    std::unordered_map<int64_t, std::unique_ptr<Request>> requests;
    std::vector<std::unique_ptr<Model>> models;
    int64_t next_id = 1;
    bool stop = false;
    std::thread scheduler, fitter;
    // statistics
    std::vector<double> latencies_ms;
    int64_t rows_done = 0, batches = 0;
    bool have_first = false;
    Clock::time_point t_first, t_last;
    std::string fatal;
};

namespace
{

void fail_request(Request *r, int code, const std::string &msg)
{
    r->status = code;
    r->error = msg;
    r->done = true;
    r->t_done = Clock::now();
}

// Creates and fits one model (synchronous on the calling thread); with
// `from` set, the fitted state is copied from that model instead of fitted.
std::unique_ptr<Model> make_model(gprat_cu_server *sv, const double *x, int64_t nx, const double *y, int64_t ny,
                                  int n_tiles, int T, int d, const double hyper[3], gprat_cu_gp *from = nullptr)
{
    auto m = std::make_unique<Model>();
    gprat_cu_gp *gp = nullptr;
    int rc = gprat_cu_gp_create(sv->device, x, nx, y, ny, n_tiles, T, d, &gp);
    if (rc != GPRAT_CU_OK)
    {
        throw Error(rc, gprat_cu_last_error());
    }
    m->gp = gp;
    m->d = d;
    if (sv->precision != GPRAT_CU_PREC_FP64)
    {
        rc = gprat_cu_gp_set_precision(gp, sv->precision);
        if (rc != GPRAT_CU_OK)
        {
            throw Error(rc, gprat_cu_last_error());
        }
    }
    if (from != nullptr)
    {
        gp_copy_fitted(gp, from);
    }
    else
    {
        gp_fit(gp, hyper, gp->stream);
    }
    gp_check(gp, gp->stream);
    // reserve a full batch: device working set, staging and pinned buffers
    gp_reserve_predict(gp, RESERVED_ROWS);
    m->d_series.ensure(static_cast<int64_t>(RESERVED_ROWS) * d);
    m->d_offsets.ensure(RESERVED_ROWS);
    m->d_mean.ensure(RESERVED_ROWS);
    m->d_var.ensure(RESERVED_ROWS);
    m->h_in.ensure(static_cast<size_t>(RESERVED_ROWS) * d * sizeof(double) + RESERVED_ROWS * sizeof(int64_t));
    m->h_out.ensure(2 * static_cast<size_t>(RESERVED_ROWS) * sizeof(double));
    GPRAT_CUDA_CHECK(cudaStreamSynchronize(gp->stream));
    m->resident = gp_resident_bytes(gp) + gp_predict_bytes(gp, RESERVED_ROWS) +
                  static_cast<int64_t>(RESERVED_ROWS) * (d + 4) * 8;
    GPRAT_CUDA_CHECK(cudaEventCreateWithFlags(&m->done_ev, cudaEventDisableTiming));
    return m;
}

// Called with the lock held: harvest finished batches.
void harvest(gprat_cu_server *sv)
{
    for (auto &mp : sv->models)
    {
        Model &md = *mp;
        if (!md.busy)
        {
            continue;
        }
        cudaError_t q = cudaEventQuery(md.done_ev);
        if (q == cudaErrorNotReady)
        {
            continue;
        }
        const Clock::time_point now = Clock::now();
        std::string err;
        int code = GPRAT_CU_OK;
        if (q != cudaSuccess)
        {
            code = GPRAT_CU_ERR_CUDA;
            err = cudaGetErrorString(q);
        }
        else
        {
            try
            {
                gp_check(md.gp, md.gp->stream);
            }
            catch (const Error &e)
            {
                code = e.code;
                err = e.what();
            }
        }
        int total = 0;
        for (Request *r : md.inflight)
        {
            total += r->m;
        }
        const double *hm = static_cast<const double *>(md.h_out.p);
        const double *hv = hm + total;
        int off = 0;
        for (Request *r : md.inflight)
        {
            if (code == GPRAT_CU_OK)
            {
                r->mean.assign(hm + off, hm + off + r->m);
                r->var.assign(hv + off, hv + off + r->m);
                r->done = true;
                r->t_done = now;
                sv->latencies_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
                sv->rows_done += r->m;
            }
            else
            {
                fail_request(r, code, err);
            }
            off += r->m;
        }
        sv->t_last = now;
        md.inflight.clear();
        sv->used -= md.inflight_bytes;
        md.inflight_bytes = 0;
        md.busy = false;
        sv->cv_done.notify_all();
        sv->cv_fit.notify_all();
    }
}

// Called with the lock held: launch one batch per idle model.  The lock is
// released while a batch is staged and enqueued (the model is marked busy
// first, so nothing else touches its buffers meanwhile).
void launch(gprat_cu_server *sv, std::unique_lock<std::mutex> &lk)
{
    for (int mi = 0; mi < static_cast<int>(sv->models.size()); ++mi)
    {
        Model &md = *sv->models[mi];
        if (md.busy)
        {
            continue;
        }
        std::vector<Request *> batch;
        int rows = 0;
        int64_t bytes = 0;
        bool anything_inflight = false;
        for (auto &o : sv->models)
        {
            anything_inflight |= o->busy;
        }
        for (auto it = sv->pending.begin(); it != sv->pending.end();)
        {
            Request *r = *it;
            if (r->model != mi)
            {
                ++it;
                continue;
            }
            // working set beyond the model's reservation
            auto extra = [&](int nrows)
            {
                return nrows <= RESERVED_ROWS ? int64_t{ 0 }
                                              : gp_predict_bytes(md.gp, nrows) - gp_predict_bytes(md.gp, RESERVED_ROWS);
            };
            const int64_t need = extra(rows + r->m) - extra(rows);
            const bool fits_rows = rows + r->m <= MAX_BATCH_ROWS || batch.empty();
            const bool fits_mem = sv->used + bytes + need <= sv->budget || (batch.empty() && !anything_inflight);
            if (!fits_rows || !fits_mem)
            {
                break;  // keep arrival order within a model
            }
            batch.push_back(r);
            rows += r->m;
            bytes += need;
            it = sv->pending.erase(it);
        }
        if (batch.empty())
        {
            continue;
        }
        md.busy = true;
        md.inflight_bytes = bytes;
        sv->used += bytes;
        sv->batches += 1;
        lk.unlock();
        int code = GPRAT_CU_OK;
        std::string err;
        try
        {
            // stage the concatenated test series and the per-row window offsets
            int64_t series_len = 0;
            for (Request *r : batch)
            {
                series_len += static_cast<int64_t>(r->series.size());
            }
            const size_t in_bytes = series_len * sizeof(double) + static_cast<size_t>(rows) * sizeof(int64_t);
            md.h_in.ensure(in_bytes);
            double *hs = static_cast<double *>(md.h_in.p);
            int64_t *ho = reinterpret_cast<int64_t *>(hs + series_len);
            int64_t pos = 0, row = 0;
            for (Request *r : batch)
            {
                std::copy(r->series.begin(), r->series.end(), hs + pos);
                for (int q = 0; q < r->m; ++q)
                {
                    ho[row++] = pos + q;
                }
                pos += static_cast<int64_t>(r->series.size());
            }
            md.d_series.ensure(series_len);
            md.d_offsets.ensure(rows);
            md.d_mean.ensure(rows);
            md.d_var.ensure(rows);
            md.h_out.ensure(2 * static_cast<size_t>(rows) * sizeof(double));
            cudaStream_t s = md.gp->stream;
            GPRAT_CUDA_CHECK(
                cudaMemcpyAsync(md.d_series.ptr, hs, series_len * sizeof(double), cudaMemcpyHostToDevice, s));
            GPRAT_CUDA_CHECK(cudaMemcpyAsync(md.d_offsets.ptr, ho, rows * sizeof(int64_t), cudaMemcpyHostToDevice, s));
            gp_predict_batch(md.gp, md.d_series.ptr, md.d_offsets.ptr, rows, md.d_mean.ptr, md.d_var.ptr, s);
            double *hout = static_cast<double *>(md.h_out.p);
            GPRAT_CUDA_CHECK(cudaMemcpyAsync(hout, md.d_mean.ptr, rows * sizeof(double), cudaMemcpyDeviceToHost, s));
            GPRAT_CUDA_CHECK(
                cudaMemcpyAsync(hout + rows, md.d_var.ptr, rows * sizeof(double), cudaMemcpyDeviceToHost, s));
            GPRAT_CUDA_CHECK(cudaEventRecord(md.done_ev, s));
        }
        catch (const Error &e)
        {
            code = e.code;
            err = e.what();
        }
        lk.lock();
        if (code == GPRAT_CU_OK)
        {
            md.inflight = std::move(batch);
        }
        else
        {
            // nothing usable was enqueued: wait for what was, then fail the batch
            cudaStreamSynchronize(md.gp->stream);
            cudaGetLastError();
            for (Request *r : batch)
            {
                fail_request(r, code, err);
            }
            sv->used -= md.inflight_bytes;
            md.inflight_bytes = 0;
            md.busy = false;
            sv->cv_done.notify_all();
        }
    }
}

void scheduler_loop(gprat_cu_server *sv)
{
    cudaSetDevice(sv->device);
    std::unique_lock<std::mutex> lk(sv->mtx);
    while (!sv->stop)
    {
        harvest(sv);
        launch(sv, lk);
        bool busy = false;
        for (auto &m : sv->models)
        {
            busy |= m->busy;
        }
        if (busy)
        {
            sv->cv_work.wait_for(lk, std::chrono::microseconds(50));
        }
        else
        {
            sv->cv_work.wait_for(lk, std::chrono::milliseconds(5),
                                 [sv] { return sv->stop || !sv->pending.empty(); });
        }
    }
    // drain: wait for in-flight batches so their buffers stay valid
    for (auto &m : sv->models)
    {
        if (m->busy)
        {
            cudaEventSynchronize(m->done_ev);
        }
    }
    harvest(sv);
}

void fitter_loop(gprat_cu_server *sv)
{
    cudaSetDevice(sv->device);
    std::unique_lock<std::mutex> lk(sv->mtx);
    while (!sv->stop)
    {
        sv->cv_fit.wait(lk, [sv] { return sv->stop || !sv->pending_fit.empty(); });
        if (sv->stop)
        {
            break;
        }
        Request *r = sv->pending_fit.front();
        // admission: a new model's resident bytes must fit next to the others
        const int64_t n = static_cast<int64_t>(r->n_tiles) * r->T;
        // (FP64 factor; the TF32/BF16 modes add a working copy, the int8 mode two digit-plane sets of 6 bytes)
        const int64_t need = n * (n + 8) * (sv->precision == GPRAT_CU_PREC_FP64        ? 8
                                            : sv->precision == GPRAT_CU_PREC_FP64_INT8 ? 20
                                                                                        : 16);
        if (sv->used + need > sv->budget)
        {
            bool inflight = false;
            for (auto &m : sv->models)
            {
                inflight |= m->busy;
            }
            if (inflight)
            {
                sv->cv_fit.wait_for(lk, std::chrono::milliseconds(2));
                continue;
            }
            sv->pending_fit.pop_front();
            fail_request(r, GPRAT_CU_ERR_OOM, "fit request exceeds the server's memory budget");
            sv->cv_done.notify_all();
            continue;
        }
        sv->pending_fit.pop_front();
        sv->used += need;
        lk.unlock();
        std::unique_ptr<Model> model;
        int code = GPRAT_CU_OK;
        std::string err;
        try
        {
            model = make_model(sv, r->x.data(), static_cast<int64_t>(r->x.size()), r->y.data(),
                               static_cast<int64_t>(r->y.size()), r->n_tiles, r->T, r->d, r->hyper);
        }
        catch (const Error &e)
        {
            code = e.code;
            err = e.what();
        }
        lk.lock();
        sv->used -= need;
        if (code == GPRAT_CU_OK)
        {
            sv->used += model->resident;
            sv->models.push_back(std::move(model));
            r->new_model = static_cast<int>(sv->models.size()) - 1;
            r->done = true;
            r->t_done = Clock::now();
        }
        else
        {
            fail_request(r, code, err);
        }
        sv->cv_done.notify_all();
        sv->cv_work.notify_all();
    }
}

template <typename F>
int guarded_sv(F &&f)
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

void need(bool c, const char *msg)
{
    if (!c)
    {
        throw Error(GPRAT_CU_ERR_INVALID_ARG, msg);
    }
}

}  // namespace

extern "C" {

int gprat_cu_server_create(int device, int64_t memory_budget_bytes, int precision, gprat_cu_server **out)
{
    return guarded_sv(
        [&]
        {
            need(out != nullptr, "server pointer must not be NULL");
            need(precision == GPRAT_CU_PREC_FP64 || precision == GPRAT_CU_PREC_MIXED_TF32 ||
                     precision == GPRAT_CU_PREC_MIXED_BF16 || precision == GPRAT_CU_PREC_FP64_INT8,
                 "unknown precision mode");
            int count = 0;
            if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
            {
                cudaGetLastError();
                throw Error(GPRAT_CU_ERR_NO_DEVICE, "Requested GPU device is not available.");
            }
            GPRAT_CUDA_CHECK(cudaSetDevice(device));
            auto sv = std::make_unique<gprat_cu_server>();
            sv->device = device;
            sv->precision = precision;
            if (memory_budget_bytes <= 0)
            {
                size_t free_b = 0, total_b = 0;
                GPRAT_CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
                memory_budget_bytes = static_cast<int64_t>(0.8 * static_cast<double>(free_b));
            }
            sv->budget = memory_budget_bytes;
            // Reserve device memory for the models up front: growing the
            // allocation pool later, while batches run, can stall a fit for
            // hundreds of milliseconds.
            sv->pool_reserved = std::min<int64_t>(memory_budget_bytes, POOL_RESERVE_MAX);
            pool_hold(sv->pool_reserved);
            gprat_cu_server *p = sv.get();
            sv->scheduler = std::thread(scheduler_loop, p);
            sv->fitter = std::thread(fitter_loop, p);
            *out = sv.release();
        });
}

int gprat_cu_server_destroy(gprat_cu_server *sv)
{
    return guarded_sv(
        [&]
        {
            if (sv == nullptr)
            {
                return;
            }
            {
                std::lock_guard<std::mutex> lk(sv->mtx);
                sv->stop = true;
            }
            sv->cv_work.notify_all();
            sv->cv_fit.notify_all();
            if (sv->scheduler.joinable())
            {
                sv->scheduler.join();
            }
            if (sv->fitter.joinable())
            {
                sv->fitter.join();
            }
            const int64_t reserved = sv->pool_reserved;
            const int dev = sv->device;
            delete sv;
            cudaSetDevice(dev);
            pool_unhold(reserved);
        });
}

int gprat_cu_server_add_model(gprat_cu_server *sv, const double *train_in, int64_t n_in, const double *train_out,
                              int64_t n_out, int n_tiles, int n_tile_size, int n_regressors, const double hyper[3],
                              int *model_id)
{
    return guarded_sv(
        [&]
        {
            need(sv != nullptr && model_id != nullptr && hyper != nullptr, "arguments must not be NULL");
            GPRAT_CUDA_CHECK(cudaSetDevice(sv->device));
            auto m = make_model(sv, train_in, n_in, train_out, n_out, n_tiles, n_tile_size, n_regressors, hyper);
            std::lock_guard<std::mutex> lk(sv->mtx);
            sv->used += m->resident;
            sv->models.push_back(std::move(m));
            *model_id = static_cast<int>(sv->models.size()) - 1;
        });
}

}  // extern "C"

namespace gprat_cu
{
// Adds to dst a copy of src's fitted model src_model (the replica layer,
// multiserve.cu): dst's handle is created from the same training data and
// tiling, then takes src's device state instead of fitting.  src_model must
// have no batch in flight.
int server_add_model_copy(gprat_cu_server *dst, gprat_cu_server *src, int src_model, const double *train_in,
                          int64_t n_in, const double *train_out, int64_t n_out, int n_tiles, int n_tile_size,
                          int n_regressors, int *model_id)
{
    return guarded_sv(
        [&]
        {
            need(dst != nullptr && src != nullptr && model_id != nullptr, "arguments must not be NULL");
            need(dst->precision == src->precision, "replicas of different precision");
            gprat_cu_gp *from = nullptr;
            {
                std::lock_guard<std::mutex> lk(src->mtx);
                need(src_model >= 0 && src_model < static_cast<int>(src->models.size()), "unknown model id");
                need(!src->models[src_model]->busy, "model has a batch in flight");
                from = src->models[src_model]->gp;
            }
            GPRAT_CUDA_CHECK(cudaSetDevice(dst->device));
            const double no_hyper[3] = { 0.0, 0.0, 0.0 };
            auto m = make_model(dst, train_in, n_in, train_out, n_out, n_tiles, n_tile_size, n_regressors, no_hyper,
                                from);
            std::lock_guard<std::mutex> lk(dst->mtx);
            dst->used += m->resident;
            dst->models.push_back(std::move(m));
            *model_id = static_cast<int>(dst->models.size()) - 1;
        });
}

// Frees a model that no request refers to and that has no batch in flight
// (replica serving drops the copies of a fit that failed on another replica):
// its device state goes back to the device and to the budget, and its id is
// never reused.
int server_release_model(gprat_cu_server *sv, int model_id)
{
    return guarded_sv(
        [&]
        {
            need(sv != nullptr, "server must not be NULL");
            Model *md = nullptr;
            {
                std::lock_guard<std::mutex> lk(sv->mtx);
                need(model_id >= 0 && model_id < static_cast<int>(sv->models.size()), "unknown model id");
                md = sv->models[model_id].get();
                need(!md->released, "model already released");
                need(!md->busy, "model has a batch in flight");
                for (const Request *r : sv->pending)
                {
                    need(r->model != model_id, "model has pending requests");
                }
                md->released = true;  // the scheduler never touches it again
                sv->used -= md->resident;
                md->resident = 0;
            }
            GPRAT_CUDA_CHECK(cudaSetDevice(sv->device));
            gprat_cu_gp *gp = md->gp;
            md->gp = nullptr;
            gprat_cu_gp_destroy(gp);
            md->d_series.release();
            md->d_mean.release();
            md->d_var.release();
            md->d_offsets.release();
        });
}

// Bytes the server's resident models hold (its admission count).
int64_t server_resident_bytes(gprat_cu_server *sv)
{
    std::lock_guard<std::mutex> lk(sv->mtx);
    return sv->used;
}
}  // namespace gprat_cu

extern "C" {

int gprat_cu_server_submit_predict(gprat_cu_server *sv, int model_id, const double *test_in, int64_t n_test_in, int m,
                                   int64_t *request_id)
{
    return guarded_sv(
        [&]
        {
            need(sv != nullptr && request_id != nullptr && test_in != nullptr, "arguments must not be NULL");
            need(m > 0, "a predict request needs at least one test point");
            auto r = std::make_unique<Request>();
            r->t_submit = Clock::now();
            r->m = m;
            r->model = model_id;
            std::lock_guard<std::mutex> lk(sv->mtx);
            need(model_id >= 0 && model_id < static_cast<int>(sv->models.size()), "unknown model id");
            need(!sv->models[model_id]->released, "model was released");
            const int d = sv->models[model_id]->d;
            need(n_test_in >= static_cast<int64_t>(m) + d - 1, "test series too short for the sliding window");
            r->series.assign(test_in, test_in + (static_cast<int64_t>(m) + d - 1));
            r->id = sv->next_id++;
            if (!sv->have_first)
            {
                sv->have_first = true;
                sv->t_first = r->t_submit;
            }
            *request_id = r->id;
            sv->pending.push_back(r.get());
            sv->requests.emplace(r->id, std::move(r));
            sv->cv_work.notify_all();
        });
}

int gprat_cu_server_submit_fit(gprat_cu_server *sv, const double *train_in, int64_t n_in, const double *train_out,
                               int64_t n_out, int n_tiles, int n_tile_size, int n_regressors, const double hyper[3],
                               int64_t *request_id)
{
    return guarded_sv(
        [&]
        {
            need(sv != nullptr && request_id != nullptr && train_in != nullptr && train_out != nullptr &&
                     hyper != nullptr,
                 "arguments must not be NULL");
            need(n_tiles > 0 && n_tile_size > 0 && n_regressors > 0, "invalid tiling");
            auto r = std::make_unique<Request>();
            r->t_submit = Clock::now();
            r->fit = true;
            r->x.assign(train_in, train_in + n_in);
            r->y.assign(train_out, train_out + n_out);
            r->n_tiles = n_tiles;
            r->T = n_tile_size;
            r->d = n_regressors;
            for (int q = 0; q < 3; ++q)
            {
                r->hyper[q] = hyper[q];
            }
            std::lock_guard<std::mutex> lk(sv->mtx);
            r->id = sv->next_id++;
            *request_id = r->id;
            sv->pending_fit.push_back(r.get());
            sv->requests.emplace(r->id, std::move(r));
            sv->cv_fit.notify_all();
        });
}

int gprat_cu_server_wait(gprat_cu_server *sv, int64_t request_id, double *mean, double *var, int *model_id,
                         double *latency_ms)
{
    return guarded_sv(
        [&]
        {
            need(sv != nullptr, "server must not be NULL");
            std::unique_lock<std::mutex> lk(sv->mtx);
            auto it = sv->requests.find(request_id);
            need(it != sv->requests.end(), "unknown request id");
            Request *r = it->second.get();
            sv->cv_done.wait(lk, [r] { return r->done; });
            std::unique_ptr<Request> owned = std::move(it->second);
            sv->requests.erase(it);
            if (r->status != GPRAT_CU_OK)
            {
                throw Error(r->status, r->error);
            }
            if (!r->fit)
            {
                if (mean != nullptr)
                {
                    std::copy(r->mean.begin(), r->mean.end(), mean);
                }
                if (var != nullptr)
                {
                    std::copy(r->var.begin(), r->var.end(), var);
                }
            }
            if (model_id != nullptr)
            {
                *model_id = r->fit ? r->new_model : r->model;
            }
            if (latency_ms != nullptr)
            {
                *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
            }
        });
}

int gprat_cu_server_stats(gprat_cu_server *sv, double *p50_ms, double *p99_ms, double *predictions_per_s,
                          int64_t *completed, int64_t *batches)
{
    return guarded_sv(
        [&]
        {
            need(sv != nullptr, "server must not be NULL");
            std::lock_guard<std::mutex> lk(sv->mtx);
            std::vector<double> l = sv->latencies_ms;
            std::sort(l.begin(), l.end());
            auto pct = [&](double q) -> double
            {
                if (l.empty())
                {
                    return 0.0;
                }
                const size_t i = std::min(l.size() - 1, static_cast<size_t>(q * static_cast<double>(l.size() - 1) + 0.5));
                return l[i];
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
                const double secs =
                    sv->have_first ? std::chrono::duration<double>(sv->t_last - sv->t_first).count() : 0.0;
                *predictions_per_s = secs > 0 ? static_cast<double>(sv->rows_done) / secs : 0.0;
            }
            if (completed != nullptr)
            {
                *completed = static_cast<int64_t>(l.size());
            }
            if (batches != nullptr)
            {
                *batches = sv->batches;
            }
        });
}

}  // extern "C"
