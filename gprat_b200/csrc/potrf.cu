// Diagonal-block Cholesky and triangular inverse in shared memory (FP64).
//
// Replaces the per-tile potrf task (LAPACKE_dpotrf2 'L',
// core/src/cpu/adapter_cblas_fp64.cpp:14-22; cusolverDnXpotrf,
// core/src/gpu/adapter_cublas.cu:9-79).  One CTA loads the lower triangle
// of a bs x bs (bs <= 128) diagonal block into shared memory, factors it
// column by column (right-looking), writes L back (the strict upper
// triangle in global memory is never touched, matching dpotrf2('L')), then
// inverts L in place by forward elimination on the identity and stores
// Linv (zero above the diagonal).  The inverse turns every later triangular
// solve against this block (panel trsm, trsv, variance solve) into a
// tensor-core GEMM.  A non-positive or NaN pivot is recorded in the status
// word (first failing global row, 1-based); the reference silently returns
// NaNs instead.
#include "common.cuh"

namespace gprat_cu
{
namespace
{

constexpr int PB = 128;         // max block size
constexpr int PS = PB + 1;      // smem row stride (conflict-free columns)
constexpr int PTHREADS = 512;

__global__ void __launch_bounds__(PTHREADS) potrf_inv_kernel(double *__restrict__ A, int64_t lda, int bs, int row0,
                                                             double *__restrict__ Linv, int64_t ldi,
                                                             DeviceStatus *__restrict__ status)
{
    extern __shared__ double sa[];  // [PB][PS] + col[PB]
    double *col = sa + PB * PS;
    const int tid = threadIdx.x;
    const int tx = tid & 31, ty = tid >> 5;
    for (int q = tid; q < bs * bs; q += PTHREADS)
    {
        int i = q / bs, c = q % bs;
        sa[i * PS + c] = (c <= i) ? A[static_cast<int64_t>(i) * lda + c] : 0.0;
    }
    __syncthreads();

    // --- Cholesky, right-looking ---------------------------------------
    __shared__ int bad;
    if (tid == 0)
    {
        bad = 0;
    }
    for (int j = 0; j < bs; ++j)
    {
        double ajj = sa[j * PS + j];
        double dj = sqrt(ajj);
        if (tid == 0 && !(ajj > 0.0) && bad == 0)
        {
            bad = row0 + j + 1;
        }
        // scale column j below the diagonal
        for (int i = j + 1 + tid; i < bs; i += PTHREADS)
        {
            sa[i * PS + j] = sa[i * PS + j] / dj;
        }
        __syncthreads();
        if (tid == 0)
        {
            sa[j * PS + j] = dj;
        }
        // rank-1 update of the trailing lower triangle (warp ty owns rows
        // j+1+ty, j+1+ty+16, ...; lanes walk the columns)
        for (int i = j + 1 + ty; i < bs; i += PTHREADS / 32)
        {
            const double lij = sa[i * PS + j];
            for (int c = j + 1 + tx; c <= i; c += 32)
            {
                sa[i * PS + c] = sa[i * PS + c] - lij * sa[c * PS + j];
            }
        }
        __syncthreads();
    }
    if (tid == 0 && bad != 0 && status != nullptr)
    {
        atomicCAS(&status->not_spd_row, 0, bad);
    }
    // write L (lower triangle incl. diagonal) back
    for (int q = tid; q < bs * bs; q += PTHREADS)
    {
        int i = q / bs, c = q % bs;
        if (c <= i)
        {
            A[static_cast<int64_t>(i) * lda + c] = sa[i * PS + c];
        }
    }
    __syncthreads();

    // --- inverse: solve L X = I in place (row p of X replaces row p of L) --
    for (int p = 0; p < bs; ++p)
    {
        double d = sa[p * PS + p];
        for (int i = p + 1 + tid; i < bs; i += PTHREADS)
        {
            col[i] = sa[i * PS + p];
        }
        // finalise row p of X: X[p][j] /= L[p][p] for j < p, X[p][p] = 1/L[p][p]
        for (int c = tid; c <= p; c += PTHREADS)
        {
            sa[p * PS + c] = (c == p) ? 1.0 / d : sa[p * PS + c] / d;
        }
        __syncthreads();
        // X[i][c] -= L[i][p] * X[p][c] for i > p, c <= p (X[i][p] starts at 0)
        for (int i = p + 1 + ty; i < bs; i += PTHREADS / 32)
        {
            const double lip = col[i];
            for (int c = tx; c <= p; c += 32)
            {
                double base = (c == p) ? 0.0 : sa[i * PS + c];
                sa[i * PS + c] = base - lip * sa[p * PS + c];
            }
        }
        __syncthreads();
    }
    for (int q = tid; q < bs * bs; q += PTHREADS)
    {
        int i = q / bs, c = q % bs;
        Linv[static_cast<int64_t>(i) * ldi + c] = (c <= i) ? sa[i * PS + c] : 0.0;
    }
}

}  // namespace

void potrf_diag(double *A, int64_t lda, int bs, int row0, double *Linv, int64_t ldi, DeviceStatus *status,
                cudaStream_t s)
{
    if (bs <= 0 || bs > PB)
    {
        throw Error(1, "potrf_diag: block size must be in [1, 128]");
    }
    constexpr size_t smem = static_cast<size_t>(PB * PS + PB) * sizeof(double);
    ensure_smem_attr(reinterpret_cast<const void *>(potrf_inv_kernel), static_cast<int>(smem));
    potrf_inv_kernel<<<1, PTHREADS, smem, s>>>(A, lda, bs, row0, Linv, ldi, status);
    GPRAT_LAUNCH_CHECK();
}

}  // namespace gprat_cu
