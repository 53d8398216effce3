// Diagonal-block Cholesky and triangular inverse in shared memory (FP64).
//
// Replaces the per-tile potrf task (LAPACKE_dpotrf2 'L',
// core/src/cpu/adapter_cblas_fp64.cpp:14-22; cusolverDnXpotrf,
// core/src/gpu/adapter_cublas.cu:9-79).  One CTA of 8 warps loads the lower
// triangle of a bs x bs (bs <= 128) diagonal block into shared memory and
// factors it in 32-wide sub-blocks:
//   1. warp 0 factors the 32 x 32 diagonal sub-block in registers (lane i
//      holds row i; column values are exchanged with shuffles) and inverts
//      it the same way (lane c holds column c of the inverse);
//   2. the rows below are solved against it with the inverse (all warps);
//   3. the trailing lower triangle is updated (all warps).
// L is written back (the strict upper triangle in global memory is never
// touched, matching dpotrf2('L')).  The full inverse Linv (zero above the
// diagonal) is then assembled block row by block row,
//   Linv_ss = X_s,  Linv_st = -X_s * sum_p L_s,p Linv_p,t,
// which turns every later triangular solve against this block (panel trsm,
// trsv, variance solve) into a tensor-core GEMM.  A non-positive or NaN
// pivot is recorded in the status word (first failing global row, 1-based);
// the reference silently returns NaNs instead.
#include "common.cuh"

namespace gprat_cu
{
namespace
{

constexpr int PB = 128;     // max block size
constexpr int PS = PB + 1;  // smem row stride of the block
constexpr int SB = 32;      // sub-block width
constexpr int XS = SB + 1;  // smem row stride of a sub-block inverse
constexpr int TS = 96 + 1;  // smem row stride of the inverse temporary
constexpr int XBLK = (SB + 1) * XS;  // one sub-block inverse plus its 1/L_ii row
constexpr int PTHREADS = 256;

// Warp 0: factor a[c0.., c0..] (w x w, w <= 32) in registers, write L back
// to smem, and store X = L^-1 (32 x 32, zero above the diagonal) in xinv.
__device__ __forceinline__ void warp_factor_invert(double *a, int c0, int w, int row0, int *bad, double *xinv)
{
    const int lane = threadIdx.x & 31;
    double r[SB];
#pragma unroll
    for (int c = 0; c < SB; ++c)
    {
        double v;
        if (lane < w && c < w)
        {
            v = (c <= lane) ? a[(c0 + lane) * PS + c0 + c] : 0.0;
        }
        else
        {
            v = (c == lane) ? 1.0 : 0.0;  // identity padding beyond w
        }
        r[c] = v;
    }
    double my_inv = 1.0;
#pragma unroll
    for (int j = 0; j < SB; ++j)
    {
        const double ajj = __shfl_sync(0xffffffffu, r[j], j);
        if (lane == 0 && j < w && !(ajj > 0.0) && *bad == 0)
        {
            *bad = row0 + c0 + j + 1;
        }
        // one reciprocal square root per pivot keeps the serial chain short
        const double inv = rsqrt(ajj);
        const double d = ajj * inv;
        if (lane == j)
        {
            r[j] = d;
            my_inv = inv;
        }
        else if (lane > j)
        {
            r[j] *= inv;
        }
#pragma unroll
        for (int c = j + 1; c < SB; ++c)
        {
            const double lcj = __shfl_sync(0xffffffffu, r[j], c);
            if (lane >= c)
            {
                r[c] -= r[j] * lcj;
            }
        }
    }
    if (lane < w)
    {
#pragma unroll
        for (int c = 0; c < SB; ++c)
        {
            if (c <= lane)
            {
                a[(c0 + lane) * PS + c0 + c] = r[c];
            }
        }
    }
    // stage 1/L_ii for the inverse, then drop r (registers) and read L from smem
    xinv[SB * XS + lane] = my_inv;
    __syncwarp();
    // inverse: lane c solves L x = e_c (column c of X); L rows are smem broadcasts
    double x[SB];
#pragma unroll
    for (int i = 0; i < SB; ++i)
    {
        double s = (i == lane) ? 1.0 : 0.0;
        const double *li = a + (c0 + i) * PS + c0;
#pragma unroll
        for (int k = 0; k < i; ++k)
        {
            s -= ((i < w) ? li[k] : 0.0) * x[k];
        }
        x[i] = s * xinv[SB * XS + i];
    }
#pragma unroll
    for (int i = 0; i < SB; ++i)
    {
        xinv[i * XS + lane] = x[i];
    }
}

__global__ void __launch_bounds__(PTHREADS) potrf_inv_kernel(double *__restrict__ A, int64_t lda, int bs, int row0,
                                                             double *__restrict__ Linv, int64_t ldi,
                                                             DeviceStatus *__restrict__ status)
{
    extern __shared__ double sa[];     // [PB][PS]
    double *xall = sa + PB * PS;       // 4 x [SB+1][XS]: sub-block inverses + 1/L_ii row
    double *tmp = xall + 4 * XBLK;     // [SB][TS]
    __shared__ int bad;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    if (tid == 0)
    {
        bad = 0;
    }
#pragma unroll 8
    for (int q = tid; q < bs * bs; q += PTHREADS)
    {
        int i = q / bs, c = q % bs;
        sa[i * PS + c] = (c <= i) ? A[static_cast<int64_t>(i) * lda + c] : 0.0;
    }
    __syncthreads();

    const int nsub = (bs + SB - 1) / SB;
    for (int s = 0; s < nsub; ++s)
    {
        const int c0 = s * SB;
        const int w = min(SB, bs - c0);
        double *xs = xall + s * XBLK;
        if (warp == 0)
        {
            warp_factor_invert(sa, c0, w, row0, &bad, xs);
        }
        __syncthreads();
        const int r0 = c0 + w;
        const int R = bs - r0;
        if (R <= 0)
        {
            break;
        }
        // panel solve: P = P X^T (4 threads per row, 8 output columns each;
        // rows in passes of PTHREADS/4, each pass reads before it writes)
        for (int pass = 0; pass * (PTHREADS / 4) < R; ++pass)
        {
            const int row = pass * (PTHREADS / 4) + (tid >> 2), grp = tid & 3;
            double v[SB];
            if (row < R)
            {
#pragma unroll
                for (int k = 0; k < SB; ++k)
                {
                    v[k] = (k < w) ? sa[(r0 + row) * PS + c0 + k] : 0.0;
                }
            }
            __syncthreads();
            if (row < R)
            {
#pragma unroll
                for (int cc = 0; cc < 8; ++cc)
                {
                    const int c = grp * 8 + cc;
                    if (c < w)
                    {
                        double acc = 0.0;
#pragma unroll
                        for (int k = 0; k < SB; ++k)
                        {
                            if (k <= c)
                            {
                                acc += v[k] * xs[c * XS + k];
                            }
                        }
                        sa[(r0 + row) * PS + c0 + c] = acc;
                    }
                }
            }
        }
        __syncthreads();
        // trailing update of the lower triangle rows/cols [r0, bs)
        for (int i = r0 + warp; i < bs; i += PTHREADS / 32)
        {
            const double *pi = sa + i * PS + c0;
            for (int c = r0 + lane; c <= i; c += 32)
            {
                const double *pc = sa + c * PS + c0;
                double acc = 0.0;
                for (int k = 0; k < w; ++k)
                {
                    acc += pi[k] * pc[k];
                }
                sa[i * PS + c] -= acc;
            }
        }
        __syncthreads();
    }
    if (tid == 0 && bad != 0 && status != nullptr)
    {
        atomicCAS(&status->not_spd_row, 0, bad);
    }
    // write L (lower triangle incl. diagonal) back
#pragma unroll 8
    for (int q = tid; q < bs * bs; q += PTHREADS)
    {
        int i = q / bs, c = q % bs;
        if (c <= i)
        {
            A[static_cast<int64_t>(i) * lda + c] = sa[i * PS + c];
        }
    }
    __syncthreads();

    // --- full inverse, block row by block row (rows < c0 already hold Linv) --
    for (int s = 0; s < nsub; ++s)
    {
        const int c0 = s * SB;
        const int w = min(SB, bs - c0);
        const double *xs = xall + s * XBLK;
        if (s > 0)
        {
            // tmp[i][j] = sum_{p=j}^{c0-1} L[c0+i][p] * Linv[p][j],  j < c0
            for (int q = tid; q < w * c0; q += PTHREADS)
            {
                const int i = q / c0, j = q % c0;
                const double *li = sa + (c0 + i) * PS;
                double acc = 0.0;
                for (int p = j; p < c0; ++p)
                {
                    acc += li[p] * sa[p * PS + j];
                }
                tmp[i * TS + j] = acc;
            }
            __syncthreads();
            // Linv[c0+i][j] = -sum_k X[i][k] tmp[k][j]
            for (int q = tid; q < w * c0; q += PTHREADS)
            {
                const int i = q / c0, j = q % c0;
                double acc = 0.0;
                for (int k = 0; k <= i; ++k)
                {
                    acc += xs[i * XS + k] * tmp[k * TS + j];
                }
                sa[(c0 + i) * PS + j] = -acc;
            }
        }
        // diagonal block: X_s
        for (int q = tid; q < w * w; q += PTHREADS)
        {
            const int i = q / w, j = q % w;
            sa[(c0 + i) * PS + c0 + j] = (j <= i) ? xs[i * XS + j] : 0.0;
        }
        __syncthreads();
    }
#pragma unroll 8
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
    constexpr size_t smem = static_cast<size_t>(PB * PS + 4 * XBLK + SB * TS) * sizeof(double);
    ensure_smem_attr(reinterpret_cast<const void *>(potrf_inv_kernel), static_cast<int>(smem));
    potrf_inv_kernel<<<1, PTHREADS, smem, s>>>(A, lda, bs, row0, Linv, ldi, status);
    GPRAT_LAUNCH_CHECK();
}

}  // namespace gprat_cu
