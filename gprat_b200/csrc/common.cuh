// Shared device/host definitions of libgprat_cuda.so (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <cstdlib>

#include <mutex>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>

namespace gprat_cu
{

// Device-resident hyper-parameter and optimiser state.  Every kernel that
// needs theta reads it from here, so an optimisation loop never returns to
// the host between steps.
struct DeviceParams
{
    double hyper[3];   // lengthscale, vertical_lengthscale, noise_variance
    double m_T[3];     // Adam first moments (SEKParams::m_T, core/include/gp_kernels.hpp:37)
    double w_T[3];     // Adam second moments (SEKParams::w_T, :39)
    double adam[4];    // learning_rate, beta1, beta2, epsilon
    int trainable[3];
    int iter;          // Adam iteration index (bias correction)
    double loss;       // last loss
    double grad[3];    // last gradient (unconstrained, reference scaling)
    double loss_hist_dummy;
};

// Device status word: first failing Cholesky pivot (1-based global row),
// and a timeout flag for bounded waits.
struct DeviceStatus
{
    int not_spd_row;  // 0 = ok
    int timeout;      // 0 = ok
};

// Error carrying a gprat_cu status code.
struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) { }
};

#define GPRAT_CUDA_CHECK(expr)                                                                              \
    do                                                                                                      \
    {                                                                                                       \
        cudaError_t _e = (expr);                                                                            \
        if (_e != cudaSuccess)                                                                              \
        {                                                                                                   \
            throw ::gprat_cu::Error(_e == cudaErrorMemoryAllocation ? 2 : 4,                                \
                                    std::string(#expr) + ": " + cudaGetErrorString(_e) + " (" __FILE__ ")"); \
        }                                                                                                   \
    } while (0)

// Counts one kernel launch of this library (stats.cu).
void note_launch();

#define GPRAT_LAUNCH_CHECK()                    \
    do                                          \
    {                                           \
        ::gprat_cu::note_launch();              \
        GPRAT_CUDA_CHECK(cudaGetLastError());   \
    } while (0)

// Step timers (stats.cu): a StepScope brackets one phase of a pipeline with
// CUDA events on its stream when gprat_cu_steps_enable(1) is in effect; the
// label is the calling entry point's prefix (StepPrefix, e.g. "predict_step")
// plus the phase ("cholesky").
bool steps_enabled();
struct StepPrefix
{
    explicit StepPrefix(const char *prefix);
    ~StepPrefix();
    StepPrefix(const StepPrefix &) = delete;
    StepPrefix &operator=(const StepPrefix &) = delete;
    std::string saved;
};
struct StepScope
{
    StepScope(const char *phase, cudaStream_t s);
    ~StepScope();
    StepScope(const StepScope &) = delete;
    StepScope &operator=(const StepScope &) = delete;
    int slot;
    cudaStream_t stream;
};

// GEMM timing hooks (stats.cu): returns true when timing is on, in which
// case the caller brackets the launch with gemm_timing_begin/end.
bool gemm_timing_enabled();
void gemm_timing_begin(cudaStream_t s);
void gemm_timing_end(cudaStream_t s, double flops);

// Programmatic dependent launch.  A kernel launched with
// programmatic_launch_attr() may start while the kernel before it in the
// stream is still running: it does its set-up (barriers, TMEM, descriptor
// prefetch), then pdl_wait() blocks until that kernel has completed and its
// memory is visible.  Every such kernel calls pdl_wait() before its first
// access to global memory; pdl_launch_dependents() (first call per CTA
// counts) lets the next kernel's set-up start once every CTA has called it
// or exited.  The next kernel's CTAs then hold SMs while they wait, so the
// kernels here signal only near their end: an early signal would let a chain
// of kernels on one stream occupy every free SM and starve other streams.
// Dependencies on events or other streams are unaffected.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

inline cudaLaunchAttribute programmatic_launch_attr()
{
    // GPRAT_CU_NO_PDL=1 launches every kernel with plain stream ordering
    static const bool off = std::getenv("GPRAT_CU_NO_PDL") != nullptr;
    cudaLaunchAttribute a = {};
    a.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    a.val.programmaticStreamSerializationAllowed = off ? 0 : 1;
    return a;
}

// Raises the dynamic shared-memory limit of `func` on the current device to
// at least `bytes` (remembers the largest limit set per kernel and device).
inline void ensure_smem_attr(const void *func, int bytes)
{
    static std::mutex mtx;
    static std::map<std::pair<const void *, int>, int> granted;
    int dev = 0;
    GPRAT_CUDA_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mtx);
    auto it = granted.find({ func, dev });
    if (it != granted.end() && it->second >= bytes)
    {
        return;
    }
    GPRAT_CUDA_CHECK(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    granted[{ func, dev }] = bytes;
}

// Writes the whole parameter block from a kernel argument (no host staging
// buffer, so back-to-back asynchronous calls cannot race on it).
void set_params(DeviceParams *p, const DeviceParams &value, cudaStream_t s);

inline int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Streaming multiprocessors of the current device.
int device_sm_count();

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// Kernel launchers (defined in the .cu files).  All matrices are row-major
// FP64 with an even leading dimension and 16-byte aligned bases.

// C[MxN] = beta*C + alpha*op(A)*op(B) on FP64 DMMA tensor cores.
//   transA=false: A is M x K (A[m*lda+k]); true: A stored K x M (A[k*lda+m]).
//   transB=false: B stored K x N (B[k*ldb+n]); true: B stored N x K (B[n*ldb+k]).
//   lower: M == N and only C[i][j] with i >= j is written (tiles above the
//          diagonal are skipped).
//   rowsq (optional, requires N <= 128): rowsq[i] += sum_j C_new[i][j]^2.
struct GemmArgs
{
    int M, N, K;
    const double *A;
    int64_t lda;
    bool transA;
    const double *B;
    int64_t ldb;
    bool transB;
    double *C;
    int64_t ldc;
    double alpha, beta;
    bool lower;
    double *rowsq;
    int k_tri;  // if >0: for C row-tile starting at row r0, the K loop starts at r0 rounded down to k_tri (A upper-triangular-by-blocks)
};
void dgemm(const GemmArgs &a, cudaStream_t s);

// SE covariance assembly (gen_tile_covariance, core/src/cpu/gp_algorithms.cpp:30-62):
// K[i][j] = v*exp(-0.5/l^2 * sum_k (x[i+k]-x[j+k])^2) (+ noise if i == j), for all
// (i,j) with floor(j/T) <= floor(i/T) (lower tiles incl. full diagonal tiles).
// K32 (optional): the same entries rounded to FP32 (row-major, ld32).
void assemble_covariance(const double *x, int n, int n_reg, int tile, const DeviceParams *p, double *K, int64_t ldk,
                         cudaStream_t s, float *K32 = nullptr, int64_t ld32 = 0);

// Cross covariance Kx[r][c] = k(xt_r, x_c), r < m, c < n
// (gen_tile_cross_covariance, core/src/cpu/gp_algorithms.cpp:113-140).  If
// alpha != nullptr, also mean[r] = sum_c Kx[r][c]*alpha[c]; if Kx == nullptr
// the matrix is not stored.
// row_offsets (optional, device, m entries): row r's window starts at
// xt[row_offsets[r]] instead of xt[r] (rows gathered from several series).
void assemble_cross(const double *xt, int m, const double *x, int n, int n_reg, const DeviceParams *p, double *Kx,
                    int64_t ldx, const double *alpha, double *mean_partial, int mean_parts, cudaStream_t s,
                    const int64_t *row_offsets = nullptr);
// Same with the matrix stored in FP32 (the mean partials stay FP64).
void assemble_cross_f32(const double *xt, int m, const double *x, int n, int n_reg, const DeviceParams *p, float *Kx,
                        int64_t ldx, const double *alpha, double *mean_partial, int mean_parts, cudaStream_t s,
                        const int64_t *row_offsets = nullptr);
// Cross covariance in FP64 (Kx, ldx) and its FP32 twin (Kx32, ld32) in one pass.
void assemble_cross_dual(const double *xt, int m, const double *x, int n, int n_reg, const DeviceParams *p,
                         double *Kx, int64_t ldx, float *Kx32, int64_t ld32, cudaStream_t s);
// mean = Kx alpha (m rows of Kx, n columns; deterministic).
void cross_times_alpha(const double *Kx, int64_t ldx, int m, int n, const double *alpha, double *mean, cudaStream_t s);
void reduce_mean(const double *mean_partial, int m, int parts, double *mean, cudaStream_t s);

// Prior covariance matrix K**[r][c] = k(xt_r, xt_c) (gen_tile_full_prior_covariance,
// core/src/cpu/gp_algorithms.cpp:64-88), full m x m.
void assemble_prior(const double *xt, int m, int n_reg, const DeviceParams *p, double *Kss, int64_t lds,
                    cudaStream_t s);

// Diagonal block Cholesky + inverse: A (bs x bs at A, lda) -> L (lower
// written back, strict upper untouched), Linv (bs x bs, ld = ldi, zero above
// the diagonal).  Records the first failing pivot in status.
void potrf_diag(double *A, int64_t lda, int bs, int row0, double *Linv, int64_t ldi, DeviceStatus *status,
                cudaStream_t s);
// Same for an FP32 block (factored in FP64 in shared memory, L written back
// in FP32 unless write_l is false); also writes Linv in FP32 (Linv32, ldi32)
// and the FP64 diagonal of L (diag, bs values).  Linv (FP64) may be null.
void potrf_diag_f32(float *A, int64_t lda, int bs, int row0, double *Linv, int64_t ldi, float *Linv32, int64_t ldi32,
                    double *diag, DeviceStatus *status, cudaStream_t s, bool write_l = true);

// Triangular solves with the blocked factor (L in Lmat, diagonal-block
// inverses in Linv, block size nb).
void trsv_forward(const double *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, double *tmp,
                  cudaStream_t s);
void trsv_backward(const double *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, double *tmp,
                   cudaStream_t s);
// Single-launch solves (trsv_fused.cu): one kernel per solve, row blocks
// claimed by ticket, every element of x written once and awaited by value.
// flags: 1 int of scratch; scratch: n doubles (the right-hand side is copied
// there).  L in FP64 or FP32; x is FP64, in place (b in, solution out).
// max_ctas > 0 bounds the grid (each CTA then solves several row blocks), so
// that the solve leaves SMs to work on another stream.
void trsv_fused_forward(const double *L, int64_t ld, const double *Linv, int n, double *x, int *flags,
                        double *scratch, DeviceStatus *st, cudaStream_t s, int max_ctas = 0);
void trsv_fused_backward(const double *L, int64_t ld, const double *Linv, int n, double *x, int *flags,
                         double *scratch, DeviceStatus *st, cudaStream_t s, int max_ctas = 0);
// skip (optional, device): when *skip != 0 at launch the solve returns at once
// (a preconditioner step of an already converged CG iteration)
void trsv_fused_forward_f32(const float *L, int64_t ld, const float *Linv, int n, double *x, int *flags,
                            double *scratch, DeviceStatus *st, cudaStream_t s, int max_ctas = 0,
                            const int *skip = nullptr);
void trsv_fused_backward_f32(const float *L, int64_t ld, const float *Linv, int n, double *x, int *flags,
                             double *scratch, DeviceStatus *st, cudaStream_t s, int max_ctas = 0,
                             const int *skip = nullptr);
// Poll budget of the single-launch solves' waits on the current device
// (polls < 0: the default, about 0.5-1 s).
void set_trsv_wait_budget(long long polls);
// Same with an FP32 factor (mixed precision); FP64 right-hand side and arithmetic.
void trsv_forward_f32(const float *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, cudaStream_t s);
void trsv_backward_f32(const float *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, cudaStream_t s);

// Loss 0.5*(y.a + sum log(L_ii^2) + n log 2pi)/n -> p->loss.
void loss_kernel(const double *y, const double *alpha, const double *L, int64_t ldl, int n, DeviceParams *p,
                 cudaStream_t s);

// var[r] = v - acc[r] (- acc2[r] when acc2 != nullptr, added to acc[r] first)
void finalize_variance(const double *acc, int m, const DeviceParams *p, double *var, cudaStream_t s,
                       const double *acc2 = nullptr);

// Fill helpers
void set_identity(double *A, int64_t lda, int n, cudaStream_t s);
void copy_rows(const double *src, int64_t lds, double *dst, int64_t ldd, int rows, int cols, cudaStream_t s);

// Adjoint: per lower tile partial sums of (Kinv - a a^T) .* dK for l and v, and
// the noise term; then reduction + Adam (see optimizer.cu).
void adjoint_trace(const double *U, int64_t ldu, const double *alpha, const double *x, int n, int n_reg,
                   const DeviceParams *p, double *partials, int *n_partials, cudaStream_t s);
void adjoint_finish(const double *partials, int n_partials, int n, DeviceParams *p, bool adam_step,
                    cudaStream_t s);

}  // namespace gprat_cu
