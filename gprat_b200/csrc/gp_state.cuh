// Device state of one GP handle (struct gprat_cu_gp of the C ABI), shared by
// the FP64 pipeline (gp.cu) and the mixed-precision pipeline (mixed.cu).
#pragma once

#include "common.cuh"
#include "gprat_cu.h"
#include "ozaki.cuh"
#include "tc_gemm.cuh"

#include <cstdint>
#include <initializer_list>
#include <string>
#include <utility>
#include <vector>

namespace gprat_cu
{

constexpr int NB = 128;   // diagonal block size (potrf + inverse)
constexpr int NBO = 512;  // outer block of the two-level factorisation and solves

// Device memory of the library's buffers.  Allocation is stream-ordered on a
// private stream of the current device (cudaMallocAsync from the device's
// default pool, then a wait on that stream only), so creating a model does
// not wait for the kernels other handles or a server have in flight, as a
// plain cudaMalloc may.  Freed memory goes back to the device (the pool keeps
// only what pool_hold reserved).  Freeing first waits for the whole device
// (the buffer may still be read by a kernel on any stream), like cudaFree.
void *device_alloc(size_t bytes);
void device_free(void *p);
// A long-lived user of the current device (a server) asks the pool to keep
// `bytes` reserved (pool_hold grows it by that much at once) and gives the
// reservation back with pool_unhold.
void pool_hold(int64_t bytes);
void pool_unhold(int64_t bytes);
// Counts the library's device allocations and frees (any handle, any
// device): a captured CUDA graph names buffer addresses, so a change of this
// count since its capture retires it.
uint64_t alloc_generation();

template <typename T>
struct DevBuf
{
    T *ptr = nullptr;
    int64_t cap = 0;  // elements
    void ensure(int64_t n)
    {
        if (n <= cap)
        {
            return;
        }
        release();
        ptr = static_cast<T *>(device_alloc(static_cast<size_t>(n) * sizeof(T)));
        cap = n;
    }
    void release()
    {
        if (ptr != nullptr)
        {
            device_free(ptr);
        }
        ptr = nullptr;
        cap = 0;
    }
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
};

// Scalars of the preconditioned CG solve on the device.
struct PcgScalars
{
    double rz;      // r . z
    double pq;      // p . q
    double rr;      // r . r
    double yy;      // y . y
    double a, b;    // step lengths
    int converged;  // 1 once |r| <= tol |y|
    int iters;      // iterations taken
};

}  // namespace gprat_cu

struct gprat_cu_gp
{
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;     // high-priority stream of the look-ahead panel factorisation
    cudaStream_t vstream = nullptr;  // low-priority stream of the variance solve beside the factorisation
    std::vector<cudaEvent_t> events;  // look-ahead ordering events (created on first use)
    // orders a device-resident call given the legacy default stream (NULL)
    // before and after the caller's work on it (created on first use)
    cudaEvent_t join_in = nullptr, join_out = nullptr;
    int n = 0, n_tiles = 0, T = 0, d = 0;
    int64_t n_in = 0;
    int64_t ld = 0;    // FP64 leading dimension
    int64_t ld32 = 0;  // FP32 / BF16 leading dimension (multiple of 64)
    int nblk = 0;
    int precision = GPRAT_CU_PREC_FP64;

    // FP64 path
    gprat_cu::DevBuf<double> x, y, K, Linv, alpha, U, partials;
    gprat_cu::DevBuf<double> xt, W, vacc, mean_part, mean, var, losses;
    gprat_cu::DevBuf<gprat_cu::DeviceParams> params;
    gprat_cu::DevBuf<gprat_cu::DeviceStatus> status;
    gprat_cu::DeviceParams *h_params = nullptr;
    gprat_cu::DeviceStatus *h_status = nullptr;

    // mixed path
    gprat_cu::DevBuf<float> K32, Linv32, W32;
    gprat_cu::DevBuf<uint16_t> Lb, Wb;  // BF16 copies (mixed-bf16)
    gprat_cu::DevBuf<double> D64;       // one diagonal block in FP64
    gprat_cu::DevBuf<double> pcg_r, pcg_z, pcg_p, pcg_q, symv_part;
    gprat_cu::DevBuf<gprat_cu::PcgScalars> pcg_s;
    int pcg_last_iters = 0;
    gprat_cu::DevBuf<int> flags;         // ticket counter of the single-launch solves
    gprat_cu::DevBuf<double> trsv_b;     // right-hand side copy of the single-launch solves

    // int8-emulated FP64 path (GPRAT_CU_PREC_FP64_INT8): digit planes of the
    // solved factor L with row exponents (A role) and block exponents (B
    // role), of the diagonal-block inverses (B role), of one unsolved panel
    // block (A role, scratch), of the solved rows of W and of one unsolved W
    // block (A role); the cross covariance kept in FP64 for the mean
    int oz_slices = 5;
    int oz_factor_groups = 0;    // digit groups kept in the factorisation's products (0 = oz_slices)
    int oz_variance_groups = 0;  // and in the variance solve's
    gprat_cu::DevBuf<int8_t> oz_lr, oz_lb, oz_inv, oz_p, oz_w, oz_wp;
    gprat_cu::DevBuf<int32_t> oz_lr_e, oz_lb_e, oz_inv_e, oz_p_e, oz_w_e, oz_wp_e;
    gprat_cu::DevBuf<double> Kx;

    // the int8-emulated fit + predict pipeline captured as one CUDA graph,
    // replayed while its key (buffers, sizes, modes, knobs) holds; graph_seen
    // is the key of the last eager run, captured when it repeats
    cudaGraphExec_t graph = nullptr;
    std::string graph_key, graph_seen;

    ~gprat_cu_gp()
    {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (stream != nullptr)
        {
            cudaStreamSynchronize(stream);
        }
        if (side != nullptr)
        {
            cudaStreamSynchronize(side);
        }
        if (vstream != nullptr)
        {
            cudaStreamSynchronize(vstream);
        }
        for (gprat_cu::DevBuf<double> *b : { &x, &y, &K, &Linv, &alpha, &U, &partials, &xt, &W, &vacc, &mean_part,
                                             &mean, &var, &losses, &D64, &pcg_r, &pcg_z, &pcg_p, &pcg_q, &symv_part, &trsv_b })
        {
            b->release();
        }
        K32.release();
        Linv32.release();
        W32.release();
        Lb.release();
        Wb.release();
        pcg_s.release();
        for (gprat_cu::DevBuf<int8_t> *b : { &oz_lr, &oz_lb, &oz_inv, &oz_p, &oz_w, &oz_wp })
        {
            b->release();
        }
        for (gprat_cu::DevBuf<int32_t> *b : { &oz_lr_e, &oz_lb_e, &oz_inv_e, &oz_p_e, &oz_w_e, &oz_wp_e })
        {
            b->release();
        }
        if (graph != nullptr)
        {
            cudaGraphExecDestroy(graph);
        }
        Kx.release();
        flags.release();
        params.release();
        status.release();
        if (h_params != nullptr)
        {
            cudaFreeHost(h_params);
        }
        if (h_status != nullptr)
        {
            cudaFreeHost(h_status);
        }
        if (side != nullptr)
        {
            cudaStreamDestroy(side);
        }
        if (vstream != nullptr)
        {
            cudaStreamDestroy(vstream);
        }
        for (cudaEvent_t e : events)
        {
            cudaEventDestroy(e);
        }
        for (cudaEvent_t e : { join_in, join_out })
        {
            if (e != nullptr)
            {
                cudaEventDestroy(e);
            }
        }
        if (stream != nullptr)
        {
            cudaStreamDestroy(stream);
        }
        if (prev >= 0)
        {
            cudaSetDevice(prev);
        }
    }
};

namespace gprat_cu
{

// mixed.cu
void factor_mixed(gprat_cu_gp *gp, cudaStream_t s,
                  const std::vector<std::pair<int, cudaEvent_t>> &splits = {});
void alpha_mixed(gprat_cu_gp *gp, cudaStream_t s, int solve_ctas = 0);
void variance_mixed(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s,
                    const int64_t *row_offsets = nullptr, int max_ctas = 0, bool recursive = true);
void fit_predict_mixed(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s);

// gp.cu: internal entry points for the serving layer (serve.cu)
void gp_fit(gprat_cu_gp *gp, const double hyper[3], cudaStream_t s);
void gp_predict_batch(gprat_cu_gp *gp, const double *d_series, const int64_t *d_row_offsets, int m, double *d_mean,
                      double *d_var, cudaStream_t s);
void gp_check(gprat_cu_gp *gp, cudaStream_t s);
int64_t gp_resident_bytes(const gprat_cu_gp *gp);
int64_t gp_predict_bytes(const gprat_cu_gp *gp, int m);
// Allocates the predict working set for m test points now (no later growth).
void gp_reserve_predict(gprat_cu_gp *gp, int m);
// Makes dst (created with the same training data, tiling and precision,
// possibly on another device) hold src's fitted state: every device buffer
// src has allocated is allocated in dst and, except the per-batch predict
// working set, copied over (peer copies across devices).  src must be idle.
// Returns the bytes copied.
int64_t gp_copy_fitted(gprat_cu_gp *dst, gprat_cu_gp *src);
void loss_mixed(gprat_cu_gp *gp, cudaStream_t s);

// mixed.cu: helpers shared by the look-ahead pipelines
// A tuning knob: the environment variable `name` if it holds an integer in
// [lo, hi], else the compiled default.
int knob(const char *name, int dflt, int lo, int hi);
// A share of the SMs in percent (knob in [10, 100]).
int sm_percent(const char *name, int dflt);
// Creates the side and variance streams and at least nevents events.
void ensure_lookahead(gprat_cu_gp *gp, int nevents);
// Events one look-ahead pipeline over n training points uses.
int lookahead_events(int n);

// ozaki_path.cu: the FP64-accurate pipeline on the int8 tensor cores
// (GPRAT_CU_PREC_FP64_INT8).  The factor is FP64 (in K, with Linv), every
// product runs as an int8-emulated FP64 GEMM, alpha comes from the FP64
// triangular solves.
void factor_oz(gprat_cu_gp *gp, cudaStream_t s, const std::vector<std::pair<int, cudaEvent_t>> &splits = {});
void variance_oz(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s,
                 const int64_t *row_offsets = nullptr, int max_ctas = 0, bool recursive = true);
void fit_predict_oz(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s);
// FP64 forward and backward solves for alpha with the FP64 factor in K.
void solve_alpha_fp64(gprat_cu_gp *gp, cudaStream_t s, int max_ctas = 0);

}  // namespace gprat_cu
