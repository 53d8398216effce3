// C-ABI entry points of libgprat_cuda.so and the device-side pipelines.
//
// A gprat_cu_gp owns, on one device: the training series and outputs, the
// covariance / Cholesky factor K (n x ld, row-major, lower triangle used),
// the inverses of its 128 x 128 diagonal blocks, alpha, the device-resident
// parameters, a status word, and grow-only workspaces (test series, the
// n_test x n solve matrix, the inverse factor for the optimiser).
//
// Pipelines (reference files in parentheses, relative to the project root):
//   factor   = SE assembly of the lower tiles + blocked right-looking
//              Cholesky: potrf+inverse of the diagonal block, panel solve as
//              a DMMA GEMM with the inverse, lower-only DMMA trailing update
//              (right_looking_cholesky_tiled, core/src/cpu/tiled_algorithms.cpp:14-57)
//   alpha    = blocked forward/backward solves (:61-115)
//   mean     = cross covariance fused with the mat-vec (:187-210)
//   variance = right-looking solve W L^T = K*  with the row sums of W^2
//              fused into the diagonal-block step (:117-149, :212-263)
//   loss     = (core/src/cpu/gp_optimizer.cpp:187-218)
//   gradient = U = L^-T, fused K^-1 = U U^T tile GEMM + derivative-tile
//              regeneration + trace reduction, then Adam (optimizer.cu)
#include "common.cuh"
#include "gp_state.cuh"
#include "gprat_cu.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <unistd.h>  // environ

using namespace gprat_cu;

namespace
{

thread_local std::string g_last_error;

struct DeviceGuard
{
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        GPRAT_CUDA_CHECK(cudaGetDevice(&prev));
        if (prev != dev)
        {
            GPRAT_CUDA_CHECK(cudaSetDevice(dev));
        }
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0)
        {
            cudaSetDevice(prev);
        }
    }
};

}  // namespace

namespace
{

template <typename F>
int guarded(F &&f)
{
    try
    {
        f();
        g_last_error.clear();
        return GPRAT_CU_OK;
    }
    catch (const Error &e)
    {
        g_last_error = e.what();
        return e.code;
    }
    catch (const std::bad_alloc &)
    {
        g_last_error = "host out of memory";
        return GPRAT_CU_ERR_OOM;
    }
    catch (const std::exception &e)
    {
        g_last_error = e.what();
        return GPRAT_CU_ERR_INVALID_ARG;
    }
}

void require(bool cond, const std::string &msg)
{
    if (!cond)
    {
        throw Error(GPRAT_CU_ERR_INVALID_ARG, msg);
    }
}

// ---------------------------------------------------------------------------
// device pipelines (enqueue only)

void upload_hyper(gprat_cu_gp *gp, const double hyper[3], cudaStream_t s)
{
    require(hyper != nullptr, "hyper-parameters must not be NULL");
    DeviceParams v;
    std::memset(&v, 0, sizeof(v));
    for (int q = 0; q < 3; ++q)
    {
        v.hyper[q] = hyper[q];
    }
    set_params(gp->params.ptr, v, s);
    GPRAT_CUDA_CHECK(cudaMemsetAsync(gp->status.ptr, 0, sizeof(DeviceStatus), s));
}

double *kblock(gprat_cu_gp *gp, int r, int c) { return gp->K.ptr + static_cast<int64_t>(r) * gp->ld + c; }

double *linv_block(gprat_cu_gp *gp, int k) { return gp->Linv.ptr + static_cast<int64_t>(k) * NB * NB; }

// C[MxN] = beta*C + alpha * A B^T (A: M x K, B: N x K, row-major)
void gemm_nt(int M, int N, int K, const double *A, int64_t lda, const double *B, int64_t ldb, double *C,
             int64_t ldc, double alpha, double beta, bool lower, double *rowsq, cudaStream_t s)
{
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.A = A;
    g.lda = lda;
    g.transA = false;
    g.B = B;
    g.ldb = ldb;
    g.transB = true;
    g.C = C;
    g.ldc = ldc;
    g.alpha = alpha;
    g.beta = beta;
    g.lower = lower;
    g.rowsq = rowsq;
    dgemm(g, s);
}

// Two-level right-looking blocked Cholesky.  Inner steps (NB = 128): FP64
// potrf + inverse of the diagonal block, panel solve P = P Linv^T (in place),
// and the update of the rest of the current outer panel.  Outer steps
// (NBO = 512): one lower-triangular DMMA update of the trailing matrix with
// K = 512.
void cholesky_blocked(gprat_cu_gp *gp, cudaStream_t s)
{
    const int n = gp->n;
    const int64_t ld = gp->ld;
    for (int K0 = 0; K0 < n; K0 += NBO)
    {
        const int bo = std::min(NBO, n - K0);
        const int pend = K0 + bo;  // end of this outer panel
        for (int r0 = K0; r0 < pend; r0 += NB)
        {
            const int bs = std::min(NB, pend - r0);
            const int k = r0 / NB;
            potrf_diag(kblock(gp, r0, r0), ld, bs, r0, linv_block(gp, k), NB, gp->status.ptr, s);
            const int rows = n - r0 - bs;
            if (rows <= 0)
            {
                continue;
            }
            // panel solve: P = P * Linv_kk^T (in place; one CTA column since bs <= 128)
            gemm_nt(rows, bs, bs, kblock(gp, r0 + bs, r0), ld, linv_block(gp, k), NB, kblock(gp, r0 + bs, r0), ld,
                    1.0, 0.0, false, nullptr, s);
            // update the rest of the outer panel: columns [r0+bs, pend)
            const int ncols = pend - (r0 + bs);
            if (ncols > 0)
            {
                // square part (rows [r0+bs, pend)): lower triangle only
                gemm_nt(ncols, ncols, bs, kblock(gp, r0 + bs, r0), ld, kblock(gp, r0 + bs, r0), ld,
                        kblock(gp, r0 + bs, r0 + bs), ld, -1.0, 1.0, true, nullptr, s);
                // rows below the outer panel
                const int below = n - pend;
                if (below > 0)
                {
                    gemm_nt(below, ncols, bs, kblock(gp, pend, r0), ld, kblock(gp, r0 + bs, r0), ld,
                            kblock(gp, pend, r0 + bs), ld, -1.0, 1.0, false, nullptr, s);
                }
            }
        }
        const int rest = n - pend;
        if (rest > 0)
        {
            // outer trailing update: C -= P_o P_o^T, K = bo, lower triangle only
            gemm_nt(rest, rest, bo, kblock(gp, pend, K0), ld, kblock(gp, pend, K0), ld, kblock(gp, pend, pend), ld,
                    -1.0, 1.0, true, nullptr, s);
        }
    }
}

// FP64 factorisation (always used by cholesky() and the optimiser).
void factor_fp64(gprat_cu_gp *gp, cudaStream_t s)
{
    {
        StepScope step("assembly", s);
        assemble_covariance(gp->x.ptr, gp->n, gp->d, gp->T, gp->params.ptr, gp->K.ptr, gp->ld, s);
    }
    StepScope step("cholesky", s);
    cholesky_blocked(gp, s);
}

// The TF32 / BF16 modes: a low-precision working copy of the factor, alpha
// refined by PCG, the variance from the low-precision factor.
bool mixed(const gprat_cu_gp *gp)
{
    return gp->precision == GPRAT_CU_PREC_MIXED_TF32 || gp->precision == GPRAT_CU_PREC_MIXED_BF16;
}

// The int8-emulated FP64 mode: an FP64 factor in K (loss and alpha as in FP64 mode).
bool int8_fp64(const gprat_cu_gp *gp) { return gp->precision == GPRAT_CU_PREC_FP64_INT8; }

// Factorisation + alpha in the handle's precision mode.
void fit(gprat_cu_gp *gp, cudaStream_t s)
{
    if (mixed(gp))
    {
        factor_mixed(gp, s);
        StepScope step("alpha refinement", s);
        alpha_mixed(gp, s);
    }
    else if (int8_fp64(gp))
    {
        factor_oz(gp, s);
        solve_alpha_fp64(gp, s);
    }
    else
    {
        factor_fp64(gp, s);
        solve_alpha_fp64(gp, s);
    }
}

// Fit, mean and variance on the handle's streams: the overlapped pipelines
// of the tensor-core modes, or fit then predict (FP64).  Used by the
// host-buffer entry points and by the device-resident one alike.
void fit_predict_var(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s);

void loss_after_fit(gprat_cu_gp *gp, cudaStream_t s)
{
    StepScope step("loss", s);
    if (mixed(gp))
    {
        loss_mixed(gp, s);
    }
    else
    {
        loss_kernel(gp->y.ptr, gp->alpha.ptr, gp->K.ptr, gp->ld, gp->n, gp->params.ptr, s);
    }
}

// Right-looking blocked solve W L^T = W (in place) over the first `rows`
// rows of W (m x ld); if rowsq != nullptr accumulates sum_j W_ij^2.
// row_limit(k) bounds the rows touched at block step k (triangular RHS).
template <typename RowLimit>
void solve_right_lt(gprat_cu_gp *gp, double *W, int64_t ldw, int rows, double *rowsq, RowLimit row_limit,
                    cudaStream_t s)
{
    // Two-level blocking like the factorisation: inner 128-column steps
    // inside a 512-column outer panel, then one K = 512 update of the rest.
    const int n = gp->n;
    const int64_t ld = gp->ld;
    for (int K0 = 0; K0 < n; K0 += NBO)
    {
        const int bo = std::min(NBO, n - K0);
        const int pend = K0 + bo;
        for (int c0 = K0; c0 < pend; c0 += NB)
        {
            const int bs = std::min(NB, pend - c0);
            const int k = c0 / NB;
            const int mrows = std::min(rows, row_limit(k));
            gemm_nt(mrows, bs, bs, W + c0, ldw, linv_block(gp, k), NB, W + c0, ldw, 1.0, 0.0, false, rowsq, s);
            const int ncols = pend - (c0 + bs);
            if (ncols > 0)
            {
                gemm_nt(mrows, ncols, bs, W + c0, ldw, kblock(gp, c0 + bs, c0), ld, W + c0 + bs, ldw, -1.0, 1.0,
                        false, nullptr, s);
            }
        }
        const int rest = n - pend;
        if (rest > 0)
        {
            const int mrows = std::min(rows, row_limit((pend - 1) / NB));
            gemm_nt(mrows, rest, bo, W + K0, ldw, kblock(gp, pend, K0), ld, W + pend, ldw, -1.0, 1.0, false, nullptr,
                    s);
        }
    }
}

// Mean (and variance if var != nullptr) for m test points at d_xt.
// row_offsets (optional, device): row r's window starts at d_xt[row_offsets[r]].
void predict_device(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s,
                    const int64_t *row_offsets = nullptr)
{
    if (m <= 0)
    {
        return;
    }
    const int parts = ceil_div(gp->n, 128);
    if (mixed(gp) && d_var != nullptr)
    {
        // a batch of separate requests (row_offsets) is served next to other
        // work: short GEMMs only
        variance_mixed(gp, d_xt, m, d_mean, d_var, s, row_offsets, 0, row_offsets == nullptr);
        return;
    }
    if (int8_fp64(gp) && d_var != nullptr)
    {
        variance_oz(gp, d_xt, m, d_mean, d_var, s, row_offsets, 0, row_offsets == nullptr);
        return;
    }
    gp->mean_part.ensure(static_cast<int64_t>(m) * parts);
    if (d_var == nullptr)
    {
        StepScope step("prediction", s);
        assemble_cross(d_xt, m, gp->x.ptr, gp->n, gp->d, gp->params.ptr, nullptr, 0, gp->alpha.ptr,
                       gp->mean_part.ptr, parts, s, row_offsets);
        reduce_mean(gp->mean_part.ptr, m, parts, d_mean, s);
        return;
    }
    gp->W.ensure(static_cast<int64_t>(m) * gp->ld);
    gp->vacc.ensure(m);
    {
        StepScope step("prediction", s);
        assemble_cross(d_xt, m, gp->x.ptr, gp->n, gp->d, gp->params.ptr, gp->W.ptr, gp->ld, gp->alpha.ptr,
                       gp->mean_part.ptr, parts, s, row_offsets);
        reduce_mean(gp->mean_part.ptr, m, parts, d_mean, s);
    }
    {
        StepScope step("forward KcK", s);
        GPRAT_CUDA_CHECK(cudaMemsetAsync(gp->vacc.ptr, 0, m * sizeof(double), s));
        solve_right_lt(gp, gp->W.ptr, gp->ld, m, gp->vacc.ptr, [m](int) { return m; }, s);
    }
    StepScope step("prediction uncertainty", s);
    finalize_variance(gp->vacc.ptr, m, gp->params.ptr, d_var, s);
}

// What a captured pipeline bakes in: buffer addresses (through the
// allocation count), sizes, the mode and the schedule's knobs (every
// GPRAT_CU_* environment variable).
std::string pipeline_key(const gprat_cu_gp *gp, const double *d_xt, int m, const double *d_mean, const double *d_var)
{
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%d|%d|%d|%d|%d|%d|%d|%p|%p|%p|%llu", gp->device, gp->n, m, gp->precision,
                  gp->oz_slices, gp->oz_factor_groups, gp->oz_variance_groups, static_cast<const void *>(d_xt),
                  static_cast<const void *>(d_mean), static_cast<const void *>(d_var),
                  static_cast<unsigned long long>(alloc_generation()));
    std::string key(buf);
    for (char **e = environ; e != nullptr && *e != nullptr; ++e)
    {
        if (std::strncmp(*e, "GPRAT_CU_", 9) == 0)
        {
            key += '|';
            key += *e;
        }
    }
    return key;
}

// The tensor-core pipelines enqueue thousands of launches on three streams
// (about 2,600 for the int8-emulated one at n = 32768).  Enqueued one by one,
// the host runs ahead of the device by the depth of the launch queue and then
// waits for room, so the variance stream's launches (enqueued after the
// factorisation's) reach the device only near the end of the factorisation,
// although the variance solve may start at its first split point.  As one
// CUDA graph a pipeline is a single launch, and the device starts every
// kernel as soon as the kernels it depends on are done (kernel nodes keep the
// priorities of the streams they were captured on).
// A run whose key equals the previous eager run's is captured and replayed
// from then on; so the buffers the graph names exist before the capture, and
// any later allocation or free changes the key.  Step and GEMM timing, which
// read their events on the host, a stream the caller is capturing, and
// GPRAT_CU_GRAPH=0 keep the eager launches.
using PipelineFn = void (*)(gprat_cu_gp *, const double *, int, double *, double *, cudaStream_t);

void fit_predict_graphed(PipelineFn run, gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var,
                         cudaStream_t s)
{
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    GPRAT_CUDA_CHECK(cudaStreamIsCapturing(s, &capturing));
    if (knob("GPRAT_CU_GRAPH", 1, 0, 1) == 0 || steps_enabled() || gemm_timing_enabled() ||
        capturing != cudaStreamCaptureStatusNone)
    {
        // (a caller capturing its stream gets the launches in its own graph)
        run(gp, d_xt, m, d_mean, d_var, s);
        return;
    }
    const std::string key = pipeline_key(gp, d_xt, m, d_mean, d_var);
    if (gp->graph_key == key)
    {
        if (gp->graph != nullptr)
        {
            GPRAT_CUDA_CHECK(cudaGraphLaunch(gp->graph, s));
        }
        else
        {
            run(gp, d_xt, m, d_mean, d_var, s);  // this key did not capture
        }
        return;
    }
    if (gp->graph_seen != key)
    {
        run(gp, d_xt, m, d_mean, d_var, s);
        gp->graph_seen = pipeline_key(gp, d_xt, m, d_mean, d_var);
        return;
    }
    if (gp->graph != nullptr)
    {
        GPRAT_CUDA_CHECK(cudaGraphExecDestroy(gp->graph));
        gp->graph = nullptr;
    }
    gp->graph_key.clear();
    cudaGraph_t g = nullptr;
    GPRAT_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try
    {
        run(gp, d_xt, m, d_mean, d_var, s);
    }
    catch (...)
    {
        cudaStreamEndCapture(s, &g);
        if (g != nullptr)
        {
            cudaGraphDestroy(g);
        }
        cudaGetLastError();
        gp->graph_seen.clear();
        throw;
    }
    GPRAT_CUDA_CHECK(cudaStreamEndCapture(s, &g));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess || pipeline_key(gp, d_xt, m, d_mean, d_var) != key)
    {
        // not replayable: this key stays eager
        if (exec != nullptr)
        {
            cudaGraphExecDestroy(exec);
        }
        cudaGetLastError();
        gp->graph_key = key;
        run(gp, d_xt, m, d_mean, d_var, s);
        return;
    }
    gp->graph = exec;
    gp->graph_key = key;
    GPRAT_CUDA_CHECK(cudaGraphLaunch(exec, s));
}

void fit_predict_var(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s)
{
    if (mixed(gp))
    {
        fit_predict_graphed(fit_predict_mixed, gp, d_xt, m, d_mean, d_var, s);
    }
    else if (int8_fp64(gp))
    {
        fit_predict_graphed(fit_predict_oz, gp, d_xt, m, d_mean, d_var, s);
    }
    else
    {
        fit(gp, s);
        predict_device(gp, d_xt, m, d_mean, d_var, s);
    }
}

void finish_and_check(gprat_cu_gp *gp)
{
    GPRAT_CUDA_CHECK(
        cudaMemcpyAsync(gp->h_status, gp->status.ptr, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, gp->stream));
    GPRAT_CUDA_CHECK(cudaStreamSynchronize(gp->stream));
    if (gp->h_status->not_spd_row != 0)
    {
        throw Error(GPRAT_CU_ERR_NOT_SPD, "Cholesky factorisation failed: covariance matrix is not positive definite "
                                          "(non-positive pivot at row " +
                                              std::to_string(gp->h_status->not_spd_row - 1) + ")");
    }
    if (gp->h_status->timeout != 0)
    {
        throw Error(GPRAT_CU_ERR_TIMEOUT, "a bounded device wait timed out");
    }
}

void upload_test(gprat_cu_gp *gp, const double *test_in, int64_t n_test_in, int m)
{
    require(test_in != nullptr, "test input must not be NULL");
    require(m >= 0, "number of test points must be >= 0");
    require(n_test_in >= static_cast<int64_t>(m) + gp->d - 1 || m == 0,
            "test input holds " + std::to_string(n_test_in) + " values; " + std::to_string(m) + " points with " +
                std::to_string(gp->d) + " regressors need " + std::to_string(static_cast<int64_t>(m) + gp->d - 1));
    const int64_t need = std::max<int64_t>(static_cast<int64_t>(m) + gp->d - 1, 1);
    gp->xt.ensure(need);
    GPRAT_CUDA_CHECK(cudaMemcpyAsync(gp->xt.ptr, test_in, (m > 0 ? need : 0) * sizeof(double), cudaMemcpyHostToDevice,
                                     gp->stream));
}

void download(gprat_cu_gp *gp, double *host, const double *dev, int64_t count)
{
    if (count > 0)
    {
        GPRAT_CUDA_CHECK(cudaMemcpyAsync(host, dev, count * sizeof(double), cudaMemcpyDeviceToHost, gp->stream));
    }
}

void gradient_device(gprat_cu_gp *gp, bool adam, cudaStream_t s)
{
    // the adjoint gradient and Adam always run in FP64
    factor_fp64(gp, s);
    solve_alpha_fp64(gp, s);
    loss_kernel(gp->y.ptr, gp->alpha.ptr, gp->K.ptr, gp->ld, gp->n, gp->params.ptr, s);
    // U = L^-T: solve U L^T = I; column block k of U has nonzeros in rows < (k+1)*NB
    gp->U.ensure(static_cast<int64_t>(gp->n) * gp->ld);
    set_identity(gp->U.ptr, gp->ld, gp->n, s);
    solve_right_lt(gp, gp->U.ptr, gp->ld, gp->n, nullptr, [](int k) { return (k + 1) * NB; }, s);
    const int t = ceil_div(gp->n, 128);
    gp->partials.ensure(static_cast<int64_t>(t) * (t + 1) / 2 * 3);
    int np = 0;
    adjoint_trace(gp->U.ptr, gp->ld, gp->alpha.ptr, gp->x.ptr, gp->n, gp->d, gp->params.ptr, gp->partials.ptr, &np,
                  s);
    adjoint_finish(gp->partials.ptr, np, gp->n, gp->params.ptr, adam, s);
}

void check_gp(gprat_cu_gp *gp) { require(gp != nullptr, "GP handle is NULL"); }

}  // namespace

namespace gprat_cu
{
// Lets other entry points of the library report through gprat_cu_last_error().
void set_last_error(const std::string &message) { g_last_error = message; }
}  // namespace gprat_cu

namespace gprat_cu
{
// Internal entry points used by the serving layer (serve.cu).
namespace
{
std::mutex g_alloc_mtx;
std::map<int, cudaStream_t> g_alloc_streams;  // per device

cudaStream_t alloc_stream(int dev)
{
    std::lock_guard<std::mutex> lk(g_alloc_mtx);
    auto it = g_alloc_streams.find(dev);
    if (it != g_alloc_streams.end())
    {
        return it->second;
    }
    cudaStream_t st = nullptr;
    GPRAT_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    g_alloc_streams[dev] = st;
    return st;
}

std::map<int, int64_t> g_pool_hold;  // bytes the device's pool keeps reserved, per device (under g_alloc_mtx)

void set_release_threshold(int dev, int64_t bytes)
{
    cudaMemPool_t pool = nullptr;
    GPRAT_CUDA_CHECK(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t keep = static_cast<uint64_t>(bytes);
    GPRAT_CUDA_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    GPRAT_CUDA_CHECK(cudaMemPoolTrimTo(pool, static_cast<size_t>(bytes)));
}
}  // namespace

// The current device's pool keeps `bytes` more reserved after frees, and is
// grown by that much now (mapping device memory into a pool can wait for the
// kernels in flight; done once up front, later allocations reuse it).
void pool_hold(int64_t bytes)
{
    int dev = 0;
    GPRAT_CUDA_CHECK(cudaGetDevice(&dev));
    int64_t total = 0;
    {
        std::lock_guard<std::mutex> lk(g_alloc_mtx);
        total = (g_pool_hold[dev] += bytes);
    }
    set_release_threshold(dev, total);
    void *p = device_alloc(static_cast<size_t>(bytes));
    device_free(p);
}

// Undoes pool_hold(bytes): the pool returns what it keeps beyond the rest.
void pool_unhold(int64_t bytes)
{
    int dev = 0;
    GPRAT_CUDA_CHECK(cudaGetDevice(&dev));
    int64_t total = 0;
    {
        std::lock_guard<std::mutex> lk(g_alloc_mtx);
        total = (g_pool_hold[dev] = std::max<int64_t>(0, g_pool_hold[dev] - bytes));
    }
    set_release_threshold(dev, total);
}

namespace
{
std::atomic<uint64_t> g_alloc_generation{ 0 };
}  // namespace

uint64_t alloc_generation() { return g_alloc_generation.load(std::memory_order_acquire); }

void *device_alloc(size_t bytes)
{
    g_alloc_generation.fetch_add(1, std::memory_order_acq_rel);
    int dev = 0;
    GPRAT_CUDA_CHECK(cudaGetDevice(&dev));
    cudaStream_t st = alloc_stream(dev);
    void *p = nullptr;
    const cudaError_t e = cudaMallocAsync(&p, bytes, st);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        throw Error(e == cudaErrorMemoryAllocation ? GPRAT_CU_ERR_OOM : GPRAT_CU_ERR_CUDA,
                    std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
                        cudaGetErrorString(e));
    }
    GPRAT_CUDA_CHECK(cudaStreamSynchronize(st));
    return p;
}

void device_free(void *p)
{
    if (p == nullptr)
    {
        return;
    }
    g_alloc_generation.fetch_add(1, std::memory_order_acq_rel);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
    {
        return;
    }
    cudaDeviceSynchronize();
    cudaStream_t st = alloc_stream(dev);
    cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
}

void gp_fit(gprat_cu_gp *gp, const double hyper[3], cudaStream_t s)
{
    upload_hyper(gp, hyper, s);
    fit(gp, s);
}

void gp_predict_batch(gprat_cu_gp *gp, const double *d_series, const int64_t *d_row_offsets, int m, double *d_mean,
                      double *d_var, cudaStream_t s)
{
    predict_device(gp, d_series, m, d_mean, d_var, s, d_row_offsets);
}

void gp_check(gprat_cu_gp *gp, cudaStream_t s)
{
    GPRAT_CUDA_CHECK(cudaMemcpyAsync(gp->h_status, gp->status.ptr, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, s));
    GPRAT_CUDA_CHECK(cudaStreamSynchronize(s));
    if (gp->h_status->not_spd_row != 0)
    {
        throw Error(GPRAT_CU_ERR_NOT_SPD, "Cholesky factorisation failed: covariance matrix is not positive definite");
    }
    if (gp->h_status->timeout != 0)
    {
        throw Error(GPRAT_CU_ERR_TIMEOUT, "a bounded device wait timed out");
    }
}

int64_t gp_resident_bytes(const gprat_cu_gp *gp)
{
    int64_t b = static_cast<int64_t>(gp->n) * gp->ld * 8 + static_cast<int64_t>(gp->nblk) * NB * NB * 8;
    if (mixed(gp))
    {
        b += static_cast<int64_t>(gp->n) * gp->ld32 * (gp->precision == GPRAT_CU_PREC_MIXED_BF16 ? 6 : 4);
    }
    else if (int8_fp64(gp))
    {
        // row and block digit planes of L, their exponents, the inverses' planes, the panel scratch
        const int64_t n = gp->n;
        b += 2 * gp->oz_slices * n * n + (n * (n / 128) + (n / 128) * (n / 128)) * 4 +
             static_cast<int64_t>(gp->oz_slices) * (gp->nblk * NB * NB + n * 128);
    }
    return b;
}

void gp_reserve_predict(gprat_cu_gp *gp, int m)
{
    DeviceGuard guard(gp->device);
    const int parts = ceil_div(gp->n, 128);
    gp->mean_part.ensure(static_cast<int64_t>(m) * parts);
    gp->vacc.ensure(2 * static_cast<int64_t>(m));
    if (gp->precision == GPRAT_CU_PREC_FP64)
    {
        gp->W.ensure(static_cast<int64_t>(m) * gp->ld);
    }
    else if (int8_fp64(gp))
    {
        const int64_t S = gp->oz_slices;
        gp->W.ensure(static_cast<int64_t>(m) * gp->ld);
        gp->oz_w.ensure(S * m * gp->n);
        gp->oz_w_e.ensure(static_cast<int64_t>(m) * (gp->n / 128));
        gp->oz_wp.ensure(S * m * 128);
        gp->oz_wp_e.ensure(m);
    }
    else
    {
        gp->W32.ensure(static_cast<int64_t>(m) * gp->ld32);
        if (gp->precision == GPRAT_CU_PREC_MIXED_BF16)
        {
            gp->Wb.ensure(static_cast<int64_t>(m) * gp->ld32);
        }
    }
}

namespace
{
// dst takes src's capacity; the contents follow unless `contents` is false.
template <typename T>
int64_t copy_buf(gprat_cu_gp *dst, DevBuf<T> &d, const gprat_cu_gp *src, const DevBuf<T> &b, bool contents)
{
    if (b.cap == 0)
    {
        return 0;
    }
    d.ensure(b.cap);
    if (!contents)
    {
        return 0;
    }
    const size_t bytes = static_cast<size_t>(b.cap) * sizeof(T);
    if (dst->device == src->device)
    {
        GPRAT_CUDA_CHECK(cudaMemcpyAsync(d.ptr, b.ptr, bytes, cudaMemcpyDeviceToDevice, dst->stream));
    }
    else
    {
        GPRAT_CUDA_CHECK(cudaMemcpyPeerAsync(d.ptr, dst->device, b.ptr, src->device, bytes, dst->stream));
    }
    return static_cast<int64_t>(bytes);
}
}  // namespace

int64_t gp_copy_fitted(gprat_cu_gp *dst, gprat_cu_gp *src)
{
    if (dst->n != src->n || dst->T != src->T || dst->d != src->d || dst->n_in != src->n_in ||
        dst->ld != src->ld || dst->ld32 != src->ld32 || dst->precision != src->precision)
    {
        throw Error(GPRAT_CU_ERR_INVALID_ARG, "model copy between handles of different shape or precision");
    }
    {
        DeviceGuard guard(src->device);
        for (cudaStream_t st : { src->stream, src->side, src->vstream })
        {
            if (st != nullptr)
            {
                GPRAT_CUDA_CHECK(cudaStreamSynchronize(st));
            }
        }
    }
    DeviceGuard guard(dst->device);
    int64_t bytes = 0;
    // fitted state: training data, factor (FP64 and low-precision copies),
    // diagonal-block inverses, alpha, parameters, status, solver scratch
    for (auto pr : { std::make_pair(&dst->x, &src->x), std::make_pair(&dst->y, &src->y),
                     std::make_pair(&dst->K, &src->K), std::make_pair(&dst->Linv, &src->Linv),
                     std::make_pair(&dst->alpha, &src->alpha), std::make_pair(&dst->U, &src->U),
                     std::make_pair(&dst->partials, &src->partials), std::make_pair(&dst->losses, &src->losses),
                     std::make_pair(&dst->D64, &src->D64), std::make_pair(&dst->pcg_r, &src->pcg_r),
                     std::make_pair(&dst->pcg_z, &src->pcg_z), std::make_pair(&dst->pcg_p, &src->pcg_p),
                     std::make_pair(&dst->pcg_q, &src->pcg_q), std::make_pair(&dst->symv_part, &src->symv_part),
                     std::make_pair(&dst->trsv_b, &src->trsv_b) })
    {
        bytes += copy_buf(dst, *pr.first, src, *pr.second, true);
    }
    bytes += copy_buf(dst, dst->K32, src, src->K32, true);
    bytes += copy_buf(dst, dst->Linv32, src, src->Linv32, true);
    bytes += copy_buf(dst, dst->Lb, src, src->Lb, true);
    bytes += copy_buf(dst, dst->pcg_s, src, src->pcg_s, true);
    // int8-emulated FP64 mode: the factor's and the inverses' digit planes
    for (auto pr : { std::make_pair(&dst->oz_lr, &src->oz_lr), std::make_pair(&dst->oz_lb, &src->oz_lb),
                     std::make_pair(&dst->oz_inv, &src->oz_inv), std::make_pair(&dst->oz_p, &src->oz_p) })
    {
        bytes += copy_buf(dst, *pr.first, src, *pr.second, true);
    }
    for (auto pr : { std::make_pair(&dst->oz_lr_e, &src->oz_lr_e), std::make_pair(&dst->oz_lb_e, &src->oz_lb_e),
                     std::make_pair(&dst->oz_inv_e, &src->oz_inv_e), std::make_pair(&dst->oz_p_e, &src->oz_p_e) })
    {
        bytes += copy_buf(dst, *pr.first, src, *pr.second, true);
    }
    dst->oz_slices = src->oz_slices;
    dst->oz_factor_groups = src->oz_factor_groups;
    dst->oz_variance_groups = src->oz_variance_groups;
    bytes += copy_buf(dst, dst->flags, src, src->flags, true);
    bytes += copy_buf(dst, dst->params, src, src->params, true);
    bytes += copy_buf(dst, dst->status, src, src->status, true);
    // per-batch predict working set: same capacity, no contents
    for (auto pr : { std::make_pair(&dst->xt, &src->xt), std::make_pair(&dst->W, &src->W),
                     std::make_pair(&dst->vacc, &src->vacc), std::make_pair(&dst->mean_part, &src->mean_part),
                     std::make_pair(&dst->mean, &src->mean), std::make_pair(&dst->var, &src->var) })
    {
        copy_buf(dst, *pr.first, src, *pr.second, false);
    }
    copy_buf(dst, dst->W32, src, src->W32, false);
    copy_buf(dst, dst->Wb, src, src->Wb, false);
    copy_buf(dst, dst->oz_w, src, src->oz_w, false);
    copy_buf(dst, dst->oz_wp, src, src->oz_wp, false);
    copy_buf(dst, dst->oz_w_e, src, src->oz_w_e, false);
    copy_buf(dst, dst->oz_wp_e, src, src->oz_wp_e, false);
    copy_buf(dst, dst->Kx, src, src->Kx, false);
    GPRAT_CUDA_CHECK(cudaStreamSynchronize(dst->stream));
    dst->pcg_last_iters = src->pcg_last_iters;
    return bytes;
}

int64_t gp_predict_bytes(const gprat_cu_gp *gp, int m)
{
    // solve matrix + mean partials + variance accumulator for m rows
    int64_t w = gp->precision == GPRAT_CU_PREC_FP64 ? static_cast<int64_t>(m) * gp->ld * 8
                                                    : static_cast<int64_t>(m) * gp->ld32 * 4;
    if (int8_fp64(gp))
    {
        // FP64 W plus its digit planes
        w = static_cast<int64_t>(m) * (gp->ld * 8 + static_cast<int64_t>(gp->oz_slices) * (gp->n + 128) + gp->n / 32 + 4);
    }
    return w + static_cast<int64_t>(m) * (ceil_div(gp->n, 128) + 2) * 8;
}
}  // namespace gprat_cu

extern "C" {

const char *gprat_cu_last_error(void) { return g_last_error.c_str(); }

const char *gprat_cu_version(void) { return "gprat_cu 0.1 sm_100a fp64-dmma"; }

int gprat_cu_device_count(int *count)
{
    return guarded(
        [&]
        {
            require(count != nullptr, "count must not be NULL");
            int c = 0;
            cudaError_t e = cudaGetDeviceCount(&c);
            if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
            {
                cudaGetLastError();
                c = 0;
            }
            else
            {
                GPRAT_CUDA_CHECK(e);
            }
            *count = c;
        });
}

int gprat_cu_gp_create(int device, const double *train_in, int64_t n_in, const double *train_out, int64_t n_out,
                       int n_tiles, int n_tile_size, int n_regressors, gprat_cu_gp **out)
{
    return guarded(
        [&]
        {
            require(out != nullptr, "output handle pointer must not be NULL");
            *out = nullptr;
            require(train_in != nullptr && train_out != nullptr, "training data must not be NULL");
            require(n_tiles > 0 && n_tile_size > 0, "n_tiles and n_tile_size must be positive");
            require(n_regressors > 0, "n_regressors must be positive");
            const int64_t n = static_cast<int64_t>(n_tiles) * n_tile_size;
            require(n <= (1LL << 30), "training set too large");
            require(n_in >= n + n_regressors - 1, "training input holds " + std::to_string(n_in) +
                                                      " values; the sliding window needs " +
                                                      std::to_string(n + n_regressors - 1));
            require(n_out >= n, "training output holds " + std::to_string(n_out) + " values; need " +
                                    std::to_string(n));
            int count = 0;
            cudaError_t ce = cudaGetDeviceCount(&count);
            if (ce != cudaSuccess || count == 0)
            {
                cudaGetLastError();
                throw Error(GPRAT_CU_ERR_NO_DEVICE, "no CUDA device available");
            }
            if (device < 0 || device >= count)
            {
                throw Error(GPRAT_CU_ERR_NO_DEVICE, "Requested GPU device is not available.");
            }
            DeviceGuard guard(device);
            auto *gp = new gprat_cu_gp();
            try
            {
                gp->device = device;
                gp->n = static_cast<int>(n);
                gp->n_tiles = n_tiles;
                gp->T = n_tile_size;
                gp->d = n_regressors;
                gp->n_in = n + n_regressors - 1;
                gp->ld = round_up(n, 8);
                gp->ld32 = round_up(n, 64);
                gp->nblk = ceil_div(n, NB);
                GPRAT_CUDA_CHECK(cudaStreamCreateWithFlags(&gp->stream, cudaStreamNonBlocking));
                GPRAT_CUDA_CHECK(cudaMallocHost(&gp->h_params, sizeof(DeviceParams)));
                GPRAT_CUDA_CHECK(cudaMallocHost(&gp->h_status, sizeof(DeviceStatus)));
                gp->params.ensure(1);
                gp->status.ensure(1);
                gp->x.ensure(gp->n_in);
                gp->y.ensure(n);
                gp->K.ensure(n * gp->ld);
                gp->Linv.ensure(static_cast<int64_t>(gp->nblk) * NB * NB);
                gp->alpha.ensure(n);
                GPRAT_CUDA_CHECK(cudaMemcpyAsync(gp->x.ptr, train_in, gp->n_in * sizeof(double),
                                                 cudaMemcpyHostToDevice, gp->stream));
                GPRAT_CUDA_CHECK(
                    cudaMemcpyAsync(gp->y.ptr, train_out, n * sizeof(double), cudaMemcpyHostToDevice, gp->stream));
                GPRAT_CUDA_CHECK(cudaMemsetAsync(gp->K.ptr, 0, n * gp->ld * sizeof(double), gp->stream));
                GPRAT_CUDA_CHECK(cudaStreamSynchronize(gp->stream));
            }
            catch (...)
            {
                delete gp;
                throw;
            }
            *out = gp;
        });
}

int gprat_cu_gp_destroy(gprat_cu_gp *gp)
{
    return guarded([&] { delete gp; });
}

int gprat_cu_gp_set_precision(gprat_cu_gp *gp, int precision)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(precision == GPRAT_CU_PREC_FP64 || precision == GPRAT_CU_PREC_MIXED_TF32 ||
                        precision == GPRAT_CU_PREC_MIXED_BF16 || precision == GPRAT_CU_PREC_FP64_INT8,
                    "unknown precision mode " + std::to_string(precision));
            require(precision == GPRAT_CU_PREC_FP64 || gp->n % NB == 0,
                    "the tensor-core precision modes need n_tiles * n_tile_size to be a multiple of 128 (got " +
                        std::to_string(gp->n) + ")");
            gp->precision = precision;
        });
}

int gprat_cu_gp_set_int8_slices(gprat_cu_gp *gp, int slices)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(slices >= OZ_MIN_SLICES && slices <= OZ_MAX_SLICES,
                    "int8 slices must be in [" + std::to_string(OZ_MIN_SLICES) + ", " + std::to_string(OZ_MAX_SLICES) +
                        "] (got " + std::to_string(slices) + ")");
            gp->oz_slices = slices;
        });
}

int gprat_cu_gp_set_int8_groups(gprat_cu_gp *gp, int factor_groups, int variance_groups)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(factor_groups >= 0 && factor_groups <= OZ_MAX_SLICES && variance_groups >= 0 &&
                        variance_groups <= OZ_MAX_SLICES,
                    "int8 digit groups must be in [0, " + std::to_string(OZ_MAX_SLICES) + "] (0 = every group)");
            gp->oz_factor_groups = factor_groups;
            gp->oz_variance_groups = variance_groups;
        });
}

int gprat_cu_cholesky(gprat_cu_gp *gp, const double hyper[3], double *tiles_out)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(tiles_out != nullptr, "output must not be NULL");
            DeviceGuard guard(gp->device);
            StepPrefix prefix("cholesky_step");
            upload_hyper(gp, hyper, gp->stream);
            factor_fp64(gp, gp->stream);
            std::vector<double> full(static_cast<size_t>(gp->n) * gp->ld);
            download(gp, full.data(), gp->K.ptr, static_cast<int64_t>(gp->n) * gp->ld);
            finish_and_check(gp);
            const int T = gp->T, nt = gp->n_tiles;
            const size_t tt = static_cast<size_t>(T) * T;
            for (int i = 0; i < nt; ++i)
            {
                for (int j = 0; j < nt; ++j)
                {
                    double *dst = tiles_out + (static_cast<size_t>(i) * nt + j) * tt;
                    if (j > i)
                    {
                        std::memset(dst, 0, tt * sizeof(double));
                        continue;
                    }
                    for (int r = 0; r < T; ++r)
                    {
                        std::memcpy(dst + static_cast<size_t>(r) * T,
                                    full.data() + static_cast<size_t>(i * T + r) * gp->ld + static_cast<size_t>(j) * T,
                                    T * sizeof(double));
                    }
                }
            }
        });
}

int gprat_cu_predict(gprat_cu_gp *gp, const double hyper[3], const double *test_in, int64_t n_test_in, int m_tiles,
                     int m_tile_size, double *mean)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(m_tiles >= 0 && m_tile_size >= 0, "m_tiles and m_tile_size must be >= 0");
            const int m = m_tiles * m_tile_size;
            require(mean != nullptr || m == 0, "mean output must not be NULL");
            DeviceGuard guard(gp->device);
            StepPrefix prefix("predict_step");
            upload_hyper(gp, hyper, gp->stream);
            upload_test(gp, test_in, n_test_in, m);
            gp->mean.ensure(std::max(m, 1));
            fit(gp, gp->stream);
            predict_device(gp, gp->xt.ptr, m, gp->mean.ptr, nullptr, gp->stream);
            download(gp, mean, gp->mean.ptr, m);
            finish_and_check(gp);
        });
}

static int predict_var_common(gprat_cu_gp *gp, const double hyper[3], const double *test_in, int64_t n_test_in,
                              int m_tiles, int m_tile_size, double *mean, double *var, const char *step_prefix)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(m_tiles >= 0 && m_tile_size >= 0, "m_tiles and m_tile_size must be >= 0");
            const int m = m_tiles * m_tile_size;
            require((mean != nullptr && var != nullptr) || m == 0, "outputs must not be NULL");
            DeviceGuard guard(gp->device);
            StepPrefix prefix(step_prefix);
            upload_hyper(gp, hyper, gp->stream);
            upload_test(gp, test_in, n_test_in, m);
            gp->mean.ensure(std::max(m, 1));
            gp->var.ensure(std::max(m, 1));
            fit_predict_var(gp, gp->xt.ptr, m, gp->mean.ptr, gp->var.ptr, gp->stream);
            download(gp, mean, gp->mean.ptr, m);
            download(gp, var, gp->var.ptr, m);
            finish_and_check(gp);
        });
}

int gprat_cu_predict_with_uncertainty(gprat_cu_gp *gp, const double hyper[3], const double *test_in,
                                      int64_t n_test_in, int m_tiles, int m_tile_size, double *mean, double *var)
{
    return predict_var_common(gp, hyper, test_in, n_test_in, m_tiles, m_tile_size, mean, var, "predict_uncer_step");
}

int gprat_cu_predict_with_full_cov(gprat_cu_gp *gp, const double hyper[3], const double *test_in, int64_t n_test_in,
                                   int m_tiles, int m_tile_size, double *mean, double *var)
{
    return predict_var_common(gp, hyper, test_in, n_test_in, m_tiles, m_tile_size, mean, var, "predict_full_cov_step");
}

int gprat_cu_predict_full_covariance(gprat_cu_gp *gp, const double hyper[3], const double *test_in,
                                     int64_t n_test_in, int m, double *mean, double *cov)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(m >= 0, "m must be >= 0");
            require((mean != nullptr && cov != nullptr) || m == 0, "outputs must not be NULL");
            DeviceGuard guard(gp->device);
            upload_hyper(gp, hyper, gp->stream);
            upload_test(gp, test_in, n_test_in, m);
            if (m == 0)
            {
                finish_and_check(gp);
                return;
            }
            gp->mean.ensure(m);
            gp->var.ensure(m);
            // the full posterior covariance is always computed in FP64
            const int saved_precision = gp->precision;
            gp->precision = GPRAT_CU_PREC_FP64;
            struct Restore
            {
                gprat_cu_gp *g;
                int p;
                ~Restore() { g->precision = p; }
            } restore{ gp, saved_precision };
            fit(gp, gp->stream);
            predict_device(gp, gp->xt.ptr, m, gp->mean.ptr, gp->var.ptr, gp->stream);
            // Sigma = K** - W W^T  (W = K* L^-T, m x n, left in gp->W)
            const int64_t lds = round_up(m, 8);
            DevBuf<double> S;
            S.ensure(static_cast<int64_t>(m) * lds);
            assemble_prior(gp->xt.ptr, m, gp->d, gp->params.ptr, S.ptr, lds, gp->stream);
            GemmArgs a{};
            a.M = m;
            a.N = m;
            a.K = gp->n;
            a.A = gp->W.ptr;
            a.lda = gp->ld;
            a.transA = false;
            a.B = gp->W.ptr;
            a.ldb = gp->ld;
            a.transB = true;
            a.C = S.ptr;
            a.ldc = lds;
            a.alpha = -1.0;
            a.beta = 1.0;
            dgemm(a, gp->stream);
            download(gp, mean, gp->mean.ptr, m);
            GPRAT_CUDA_CHECK(cudaMemcpy2DAsync(cov, m * sizeof(double), S.ptr, lds * sizeof(double),
                                               m * sizeof(double), m, cudaMemcpyDeviceToHost, gp->stream));
            finish_and_check(gp);
            S.release();
        });
}

int gprat_cu_compute_loss(gprat_cu_gp *gp, const double hyper[3], double *loss)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(loss != nullptr, "loss must not be NULL");
            DeviceGuard guard(gp->device);
            upload_hyper(gp, hyper, gp->stream);
            fit(gp, gp->stream);
            loss_after_fit(gp, gp->stream);
            GPRAT_CUDA_CHECK(cudaMemcpyAsync(gp->h_params, gp->params.ptr, sizeof(DeviceParams),
                                             cudaMemcpyDeviceToHost, gp->stream));
            finish_and_check(gp);
            *loss = gp->h_params->loss;
        });
}

int gprat_cu_loss_grad(gprat_cu_gp *gp, const double hyper[3], double *loss, double grad[3])
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(loss != nullptr && grad != nullptr, "outputs must not be NULL");
            DeviceGuard guard(gp->device);
            upload_hyper(gp, hyper, gp->stream);
            gradient_device(gp, false, gp->stream);
            GPRAT_CUDA_CHECK(cudaMemcpyAsync(gp->h_params, gp->params.ptr, sizeof(DeviceParams),
                                             cudaMemcpyDeviceToHost, gp->stream));
            finish_and_check(gp);
            *loss = gp->h_params->loss;
            for (int q = 0; q < 3; ++q)
            {
                grad[q] = gp->h_params->grad[q];
            }
        });
}

static void upload_opt_state(gprat_cu_gp *gp, const double params[9], const double adam[4], const int trainable[3],
                             int iter)
{
    require(params != nullptr && adam != nullptr && trainable != nullptr, "optimiser arguments must not be NULL");
    require(iter >= 0, "iter must be >= 0");
    DeviceParams v;
    std::memset(&v, 0, sizeof(v));
    for (int q = 0; q < 3; ++q)
    {
        v.hyper[q] = params[q];
        v.m_T[q] = params[3 + q];
        v.w_T[q] = params[6 + q];
        v.trainable[q] = trainable[q] != 0;
    }
    for (int q = 0; q < 4; ++q)
    {
        v.adam[q] = adam[q];
    }
    v.iter = iter;
    set_params(gp->params.ptr, v, gp->stream);
    GPRAT_CUDA_CHECK(cudaMemsetAsync(gp->status.ptr, 0, sizeof(DeviceStatus), gp->stream));
}

static void download_opt_state(gprat_cu_gp *gp, double params[9])
{
    GPRAT_CUDA_CHECK(
        cudaMemcpyAsync(gp->h_params, gp->params.ptr, sizeof(DeviceParams), cudaMemcpyDeviceToHost, gp->stream));
    finish_and_check(gp);
    for (int q = 0; q < 3; ++q)
    {
        params[q] = gp->h_params->hyper[q];
        params[3 + q] = gp->h_params->m_T[q];
        params[6 + q] = gp->h_params->w_T[q];
    }
}

int gprat_cu_optimize_step(gprat_cu_gp *gp, double params[9], const double adam[4], const int trainable[3], int iter,
                           double *loss)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(loss != nullptr, "loss must not be NULL");
            DeviceGuard guard(gp->device);
            upload_opt_state(gp, params, adam, trainable, iter);
            gradient_device(gp, true, gp->stream);
            download_opt_state(gp, params);
            *loss = gp->h_params->loss;
        });
}

int gprat_cu_optimize(gprat_cu_gp *gp, double params[9], const double adam[4], const int trainable[3], int opt_iter,
                      double *losses)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(opt_iter >= 0, "opt_iter must be >= 0");
            require(losses != nullptr || opt_iter == 0, "losses must not be NULL");
            DeviceGuard guard(gp->device);
            upload_opt_state(gp, params, adam, trainable, 0);
            gp->losses.ensure(std::max(opt_iter, 1));
            for (int it = 0; it < opt_iter; ++it)
            {
                gradient_device(gp, true, gp->stream);
                GPRAT_CUDA_CHECK(cudaMemcpyAsync(gp->losses.ptr + it, &gp->params.ptr->loss, sizeof(double),
                                                 cudaMemcpyDeviceToDevice, gp->stream));
            }
            download(gp, losses, gp->losses.ptr, opt_iter);
            download_opt_state(gp, params);
        });
}

int gprat_cu_fit_predict_device(gprat_cu_gp *gp, const double hyper[3], const double *d_test_in, int64_t n_test_in,
                                int m, double *d_mean, double *d_var, void *stream)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(m >= 0, "m must be >= 0");
            require(d_test_in != nullptr && d_mean != nullptr, "device buffers must not be NULL");
            require(n_test_in >= static_cast<int64_t>(m) + gp->d - 1, "test series too short for the sliding window");
            DeviceGuard guard(gp->device);
            // NULL is the legacy default stream: the work runs on the handle's
            // own (non-blocking) stream, ordered after the work already on the
            // default stream and before the work enqueued on it later
            const bool legacy = stream == nullptr;
            cudaStream_t s = legacy ? gp->stream : static_cast<cudaStream_t>(stream);
            if (legacy)
            {
                for (cudaEvent_t *e : { &gp->join_in, &gp->join_out })
                {
                    if (*e == nullptr)
                    {
                        GPRAT_CUDA_CHECK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
                    }
                }
                GPRAT_CUDA_CHECK(cudaEventRecord(gp->join_in, cudaStreamLegacy));
                GPRAT_CUDA_CHECK(cudaStreamWaitEvent(s, gp->join_in, 0));
            }
            upload_hyper(gp, hyper, s);
            if (d_var != nullptr)
            {
                // the schedule gprat_cu_predict_with_uncertainty runs
                fit_predict_var(gp, d_test_in, m, d_mean, d_var, s);
            }
            else
            {
                fit(gp, s);
                predict_device(gp, d_test_in, m, d_mean, nullptr, s);
            }
            if (legacy)
            {
                GPRAT_CUDA_CHECK(cudaEventRecord(gp->join_out, s));
                GPRAT_CUDA_CHECK(cudaStreamWaitEvent(cudaStreamLegacy, gp->join_out, 0));
            }
        });
}

int gprat_cu_gp_pcg_iterations(gprat_cu_gp *gp, int *iterations)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            require(iterations != nullptr, "iterations must not be NULL");
            *iterations = 0;
            if (mixed(gp) && gp->pcg_s.ptr != nullptr)
            {
                // the solve's counter lives on the device (no host wait inside the solve)
                DeviceGuard guard(gp->device);
                PcgScalars h{};
                GPRAT_CUDA_CHECK(cudaDeviceSynchronize());
                GPRAT_CUDA_CHECK(cudaMemcpy(&h, gp->pcg_s.ptr, sizeof(PcgScalars), cudaMemcpyDeviceToHost));
                gp->pcg_last_iters = h.iters;
                *iterations = h.iters;
            }
        });
}

int gprat_cu_check_status(gprat_cu_gp *gp)
{
    return guarded(
        [&]
        {
            check_gp(gp);
            DeviceGuard guard(gp->device);
            GPRAT_CUDA_CHECK(cudaDeviceSynchronize());
            finish_and_check(gp);
        });
}

}  // extern "C"
