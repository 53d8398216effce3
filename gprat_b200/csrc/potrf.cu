// Diagonal-block Cholesky and triangular inverse in shared memory (FP64).
//
// Replaces the per-tile potrf task (LAPACKE_dpotrf2 'L',
// core/src/cpu/adapter_cblas_fp64.cpp:14-22; cusolverDnXpotrf,
// core/src/gpu/adapter_cublas.cu:9-79).  One CTA of 8 warps factors a
// bs x bs (bs <= 128) diagonal block; a block smaller than 128 is padded with
// the identity, so every loop below has a fixed trip count.  Right-looking in
// 32-wide sub-blocks s = 0..3:
//   1. warp 0 factors the 32 x 32 diagonal sub-block in registers (lane i
//      holds row i; the pivot travels by shuffle, the new column of L through
//      shared memory; branch-free) and forms its inverse X_s column by column
//      (lane c solves L x = e_c in axpy order, so the 31 updates of a step are
//      independent);
//   2. panel solve P = A_rs X_s^T and trailing update A_rr -= P P^T on the
//      FP64 tensor cores (mma.sync m16n8k8 f64; upper-triangular zero blocks
//      of X_s are skipped);
// and the full inverse is assembled block row by block row on the tensor
// cores,  Linv_s,<s = -X_s (L_s,<s Linv_<s,<s),  Linv_ss = X_s,
// which turns every later triangular solve against this block (panel trsm,
// trsv, variance solve) into a GEMM.  Row block s is assembled by warps 1-7
// while warp 0 runs the pivot chain of sub-block s+1 (the two touch disjoint
// rows, and no later step reads rows above the current sub-block), so only
// the last row block's assembly follows the factorisation; each row block of
// L is written back before its assembly replaces it.  L is written back to the lower
// triangle only (the strict upper triangle in global memory is never
// touched, matching dpotrf2('L')).  A non-positive or NaN pivot is recorded
// in the status word (first failing global row, 1-based); the reference
// silently returns NaNs instead.
#include "common.cuh"

namespace gprat_cu
{
namespace
{

constexpr int PB = 128;                   // block size (padded)
constexpr int PS = PB + 4;                // smem row stride of the block (conflict-free fragment loads)
constexpr int SB = 32;                    // sub-block width
constexpr int XS = SB + 4;                // smem row stride of a sub-block inverse
constexpr int TS = 3 * SB + 4;            // smem row stride of the assembly temporary
constexpr int PTHREADS = 256;
constexpr int NWARPS = PTHREADS / 32;
constexpr size_t SMEM_DOUBLES = PB * PS + 4 * SB * XS + PB + SB * TS + 2 * SB;

template <typename T>
struct PairOf;
template <>
struct PairOf<double>
{
    using type = double2;
};
template <>
struct PairOf<float>
{
    using type = float2;
};

__device__ __forceinline__ void dmma(double (&c)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Fragment loads from row-major shared matrices (g = lane / 4, t = lane % 4).
// A: rows m0.., k-columns k0..
__device__ __forceinline__ void frag_a(double (&a)[4], const double *M, int ld, int m0, int k0, int g, int t)
{
    a[0] = M[(m0 + g) * ld + k0 + t];
    a[1] = M[(m0 + g + 8) * ld + k0 + t];
    a[2] = M[(m0 + g) * ld + k0 + t + 4];
    a[3] = M[(m0 + g + 8) * ld + k0 + t + 4];
}
// B = M^T with M row-major (N x K): B[k][n] = M[n][k]
__device__ __forceinline__ void frag_bt(double (&b)[2], const double *M, int ld, int n0, int k0, int g, int t)
{
    b[0] = M[(n0 + g) * ld + k0 + t];
    b[1] = M[(n0 + g) * ld + k0 + t + 4];
}
// B row-major (K x N)
__device__ __forceinline__ void frag_b(double (&b)[2], const double *M, int ld, int n0, int k0, int g, int t)
{
    b[0] = M[(k0 + t) * ld + n0 + g];
    b[1] = M[(k0 + t + 4) * ld + n0 + g];
}

// Warp 0: factor the 32 x 32 sub-block at (c0, c0), write L back to smem,
// and store the pivot reciprocals 1/L_jj in dinv[0..31].
//
// Lane i keeps row i in registers; fully unrolled, so every register index is
// a compile-time constant and pivot j updates exactly the columns j+1..31.
// Branch-free: a lane's entries above the diagonal receive values that are
// never read, which keeps the warp converged (per-lane conditional updates
// compile to divergent branches that cost more than the arithmetic).
// colbuf (2 x 32 doubles, alternating by pivot, so one __syncwarp per pivot
// suffices) broadcasts the new column of L; the update reads it in pairs.
// The next pivot's lane computes its updated diagonal a_j+1,j+1 - l^2 from its
// own l before the broadcast, and the next pivot's shuffle and rsqrt are
// issued before the column update, so their latency overlaps it.
__device__ __forceinline__ void diag_factor_invert(double *a, int c0, int bs, int row0, int *bad, double *dinv,
                                                   double *colbuf)
{
    const int lane = threadIdx.x & 31;
    double r[SB];  // r[c] = A[lane][c0 + c]
    {
        const double *arow = a + (c0 + lane) * PS + c0;
#pragma unroll
        for (int c = 0; c < SB; ++c)
        {
            r[c] = (c <= lane) ? arow[c] : 0.0;
        }
    }
    int first_bad = 0;
    double ajj = __shfl_sync(0xffffffffu, r[0], 0);  // the current pivot's updated diagonal entry
    double inv = rsqrt(ajj);
#pragma unroll
    for (int j = 0; j < SB; ++j)
    {
        double *cb = colbuf + (j & 1) * SB;
        first_bad = (first_bad == 0 && !(ajj > 0.0) && c0 + j < bs) ? row0 + c0 + j + 1 : first_bad;
        const double l = (lane == j) ? ajj * inv : r[j] * inv;  // L[lane][j] for lane >= j
        cb[lane] = l;
        a[(c0 + lane) * PS + c0 + j] = l;  // above the diagonal: a value nobody reads
        if (lane == 0)
        {
            dinv[j] = inv;
        }
        if (j + 1 < SB)
        {
            const double dnext = r[j + 1] - l * l;  // lane j+1: the next pivot
            __syncwarp();
            // the next pivot's shuffle and rsqrt are independent of the column
            // update below and overlap it
            ajj = __shfl_sync(0xffffffffu, dnext, j + 1);
            inv = rsqrt(ajj);
            int c = j + 1;
            if (c & 1)
            {
                r[c] -= l * cb[c];
                ++c;
            }
#pragma unroll
            for (; c < SB; c += 2)
            {
                const double2 v = *reinterpret_cast<const double2 *>(cb + c);
                r[c] -= l * v.x;
                r[c + 1] -= l * v.y;
            }
        }
    }
    if (lane == 0 && first_bad != 0 && *bad == 0)
    {
        *bad = first_bad;
    }
}

// All 8 warps: X = L^-1 of the factored 32 x 32 sub-block at (c0, c0), zero
// above the diagonal, into xinv.  Warp w solves columns 4w .. 4w+3; lane i owns
// row i and the four columns' x_i.  The system is scaled to a unit diagonal
// first (row i of L and of the right-hand side times 1/L_ii), so step k is one
// shuffle of the final x_k and one FMA on the lanes below (their strictly
// lower entries; every other coefficient is zero).  Fully unrolled (32 short
// steps) and branch-free.
__device__ __forceinline__ void diag_inverse_all_warps(const double *a, int c0, const double *dinv, double *xinv)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double lrow[SB];
    const double *arow = a + (c0 + lane) * PS + c0;
    const double di = dinv[lane];
#pragma unroll
    for (int c = 0; c < SB; ++c)
    {
        lrow[c] = (c < lane) ? arow[c] * di : 0.0;
    }
    double x[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        x[q] = (lane == 4 * warp + q) ? di : 0.0;
    }
#pragma unroll
    for (int k = 0; k < SB; ++k)
    {
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            const double xk = __shfl_sync(0xffffffffu, x[q], k);
            x[q] -= lrow[k] * xk;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        xinv[lane * XS + 4 * warp + q] = x[q];
    }
}

__device__ __forceinline__ void cp_async16_zfill(void *smem, const void *gmem, int bytes)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gmem), "r"(bytes) : "memory");
}

// Offset (in 16-byte chunks) of row i in the packed FP32 staging of a lower
// triangle whose row r holds r / 4 + 1 chunks (columns 0 .. 4 (r / 4) + 3).
__device__ __forceinline__ int staged_row_chunks(int i)
{
    const int q = i >> 2, r = i & 3;
    return (q + 1) * (2 * q + r);
}

// Loads the lower triangle of the block (rows < bs) with 16-byte cp.async
// copies, then pads: the strict upper triangle is zero and rows >= bs are
// identity rows.  Needs A and lda * sizeof(T) 16-byte aligned.  Every copy
// stops at column i of its row (the rest of the chunk is zero-filled), so
// nothing right of the block's diagonal is read.
//   FP64: rows go straight to their place in sa;
//   FP32: rows are packed into `stage` (2112 chunks, 33 KB), then widened.
template <typename T>
__device__ __forceinline__ void load_lower_async(const T *__restrict__ A, int64_t lda, int bs, double *sa,
                                                 double *stage)
{
    constexpr int CH = 16 / sizeof(T);  // elements per chunk
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *st32 = reinterpret_cast<float *>(stage);
    for (int i = warp; i < bs; i += NWARPS)
    {
        const int nchunks = i / CH + 1;
        for (int k = lane; k < nchunks; k += 32)
        {
            const int c = k * CH;
            const int bytes = min(CH, i + 1 - c) * static_cast<int>(sizeof(T));
            void *dst = (sizeof(T) == 8) ? static_cast<void *>(sa + i * PS + c)
                                         : static_cast<void *>(st32 + 4 * (staged_row_chunks(i) + k));
            cp_async16_zfill(dst, A + static_cast<int64_t>(i) * lda + c, bytes);
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    for (int q = threadIdx.x; q < PB * PB / 2; q += PTHREADS)
    {
        const int i = q >> 6, c = 2 * (q & 63);
        double v0 = (i == c) ? 1.0 : 0.0, v1 = (i == c + 1) ? 1.0 : 0.0;
        if (i < bs && c <= i)
        {
            if (sizeof(T) == 8)
            {
                const double2 w = *reinterpret_cast<const double2 *>(sa + i * PS + c);
                v0 = w.x;
                v1 = (c + 1 <= i) ? w.y : 0.0;
            }
            else
            {
                const float *row = st32 + 4 * staged_row_chunks(i);
                v0 = static_cast<double>(row[c]);
                v1 = (c + 1 <= i) ? static_cast<double>(row[c + 1]) : 0.0;
            }
        }
        *reinterpret_cast<double2 *>(sa + i * PS + c) = make_double2(v0, v1);
    }
}

// Barrier over the nthreads threads of warps first .. (a named barrier; id 0
// with every thread is __syncthreads).
__device__ __forceinline__ void bar_sync(int id, int nthreads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Inverse of row block s (rows 32s .. 32s + 31), in place in sa, whose rows
// < 32s already hold Linv:  Linv_s,<s = -X_s (L_s,<s Linv_<s,<s),  Linv_ss = X_s.
// Run by nwarps warps starting at first_warp; barrier bar_id (over those
// warps) separates the reads of L_s,<s from the writes that replace it.
__device__ __forceinline__ void assemble_row_block(double *sa, const double *xs, double *tbuf, int s, int first_warp,
                                                   int nwarps, int bar_id)
{
    const int lane = threadIdx.x & 31, w = (threadIdx.x >> 5) - first_warp;
    const int g = lane >> 2, t = lane & 3;
    const int c0 = s * SB;
    if (s > 0)
    {
        // T = L[c0.., 0..c0) Linv[0..c0, 0..c0)   (32 x c0; Linv lower: k >= n)
        const int nt_count = c0 / 8;
        for (int tile = w; tile < 2 * nt_count; tile += nwarps)
        {
            const int mi = tile / nt_count, nt = tile % nt_count;
            double cf[4] = { 0.0, 0.0, 0.0, 0.0 };
            for (int kk = nt; kk < nt_count; ++kk)
            {
                double af[4], bf[2];
                frag_a(af, sa, PS, c0 + 16 * mi, 8 * kk, g, t);
                frag_b(bf, sa, PS, 8 * nt, 8 * kk, g, t);
                dmma(cf, af, bf);
            }
            double *c = tbuf + (16 * mi + g) * TS + 8 * nt + 2 * t;
            c[0] = cf[0];
            c[1] = cf[1];
            c[8 * TS] = cf[2];
            c[8 * TS + 1] = cf[3];
        }
        bar_sync(bar_id, nwarps * 32);
        // Linv[c0.., 0..c0) = -X T   (X lower: k <= row)
        for (int tile = w; tile < 2 * nt_count; tile += nwarps)
        {
            const int mi = tile / nt_count, nt = tile % nt_count;
            double cf[4] = { 0.0, 0.0, 0.0, 0.0 };
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
            {
                if (kk <= 2 * mi + 1)
                {
                    double af[4], bf[2];
                    frag_a(af, xs, XS, 16 * mi, 8 * kk, g, t);
                    frag_b(bf, tbuf, TS, 8 * nt, 8 * kk, g, t);
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                    {
                        af[e] = -af[e];
                    }
                    dmma(cf, af, bf);
                }
            }
            double *c = sa + (c0 + 16 * mi + g) * PS + 8 * nt + 2 * t;
            c[0] = cf[0];
            c[1] = cf[1];
            c[8 * PS] = cf[2];
            c[8 * PS + 1] = cf[3];
        }
    }
    // diagonal block: X_s (zero above the diagonal)
    for (int q = w * 32 + lane; q < SB * SB; q += nwarps * 32)
    {
        const int i = q / SB, j = q % SB;
        sa[(c0 + i) * PS + c0 + j] = (j <= i) ? xs[i * XS + j] : 0.0;
    }
}

// Writes row block c0 .. c0 + 31 of L (lower triangle with the diagonal, rows
// < bs) back to A: in pairs of columns when the block is 16-byte aligned,
// else element by element.
template <typename T>
__device__ __forceinline__ void write_l_block(T *A, int64_t lda, const double *sa, int c0, int bs, bool aligned)
{
    using Pair = typename PairOf<T>::type;
    for (int q = threadIdx.x; q < SB * (PB / 2); q += PTHREADS)
    {
        const int i = c0 + (q >> 6), c = 2 * (q & 63);
        if (i >= bs || c > i)
        {
            continue;
        }
        T *dst = A + static_cast<int64_t>(i) * lda + c;
        if (aligned)
        {
            const double2 v = *reinterpret_cast<const double2 *>(sa + i * PS + c);
            if (c + 1 <= i)
            {
                Pair w;
                w.x = static_cast<T>(v.x);
                w.y = static_cast<T>(v.y);
                *reinterpret_cast<Pair *>(dst) = w;
            }
            else
            {
                dst[0] = static_cast<T>(v.x);
            }
        }
        else
        {
            dst[0] = static_cast<T>(sa[i * PS + c]);
            if (c + 1 <= i)
            {
                dst[1] = static_cast<T>(sa[i * PS + c + 1]);
            }
        }
    }
}

// True when the block and its rows start on 16-byte boundaries.
template <typename T>
__device__ __forceinline__ bool aligned16(const T *A, int64_t lda)
{
    return ((reinterpret_cast<uintptr_t>(A) | static_cast<uintptr_t>(lda * sizeof(T))) & 15) == 0;
}

// T: element type of the block in global memory (FP64, or FP32 for the
// mixed path, which then also receives Linv in FP32 and the FP64 diagonal of L).
template <typename T>
__global__ void __launch_bounds__(PTHREADS, 1) potrf_inv_kernel(T *__restrict__ A, int64_t lda, int bs, int row0,
                                                                double *__restrict__ Linv, int64_t ldi,
                                                                float *__restrict__ Linv32, int64_t ldi32,
                                                                double *__restrict__ diag_out,
                                                                DeviceStatus *__restrict__ status, int write_l)
{
    extern __shared__ double sa[];  // [PB][PS]
    double *xall = sa + PB * PS;    // 4 x [SB][XS] sub-block inverses
    double *dinv = xall + 4 * SB * XS;       // [PB] pivot reciprocals
    double *tbuf = dinv + PB;                // [SB][TS]
    double *colbuf = tbuf + SB * TS;         // [2][SB] column broadcast of the diagonal factorisation
    __shared__ int bad;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    if (tid == 0)
    {
        bad = 0;
    }
    pdl_wait();  // the previous kernel's results are visible from here on
    if (aligned16(A, lda))
    {
        load_lower_async(A, lda, bs, sa, xall);
    }
    else
    {
        // unaligned block: element loads of the lower triangle, identity padding
        for (int q = tid; q < PB * PB; q += PTHREADS)
        {
            const int i = q >> 7, c = q & (PB - 1);
            sa[i * PS + c] = (i < bs && c <= i) ? static_cast<double>(A[static_cast<int64_t>(i) * lda + c])
                                                : ((i == c) ? 1.0 : 0.0);
        }
    }
    __syncthreads();

    const bool al = aligned16(A, lda);
#pragma unroll 1
    for (int s = 0; s < 4; ++s)
    {
        const int c0 = s * SB;
        double *xs = xall + s * SB * XS;
        if (warp == 0)
        {
            diag_factor_invert(sa, c0, bs, row0, &bad, dinv + c0, colbuf);
        }
        else if (s > 0)
        {
            // the previous row block's inverse, beside this sub-block's pivots
            // (disjoint rows; later steps never read rows above c0)
            assemble_row_block(sa, xall + (s - 1) * SB * XS, tbuf, s - 1, 1, NWARPS - 1, 1);
        }
        __syncthreads();
        diag_inverse_all_warps(sa, c0, dinv + c0, xs);
        // row block s of L is final: write it back (and its diagonal) before
        // the assembly replaces it with Linv
        if (write_l)
        {
            write_l_block(A, lda, sa, c0, bs, al);
        }
        if (diag_out != nullptr && tid < SB && c0 + tid < bs)
        {
            diag_out[c0 + tid] = sa[(c0 + tid) * PS + c0 + tid];
        }
        __syncthreads();
        if (s == 3)
        {
            break;
        }
        const int r0 = c0 + SB;
        const int R = PB - r0;  // 96, 64, 32 rows below
        // panel: P = A[r0.., c0..c0+31] X^T  (warp w owns rows r0 + 16w .. +15)
        if (warp < R / 16)
        {
            const int m0 = r0 + 16 * warp;
            double af[4][4];
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
            {
                frag_a(af[kk], sa, PS, m0, c0 + 8 * kk, g, t);
            }
            double cf[4][4];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt)
            {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                {
                    cf[nt][e] = 0.0;
                }
#pragma unroll
                for (int kk = 0; kk <= nt; ++kk)  // X^T is zero where k > n
                {
                    double bf[2];
                    frag_bt(bf, xs, XS, 8 * nt, 8 * kk, g, t);
                    dmma(cf[nt], af[kk], bf);
                }
            }
            __syncwarp();
#pragma unroll
            for (int nt = 0; nt < 4; ++nt)
            {
                double *c = sa + (m0 + g) * PS + c0 + 8 * nt + 2 * t;
                c[0] = cf[nt][0];
                c[1] = cf[nt][1];
                c[8 * PS] = cf[nt][2];
                c[8 * PS + 1] = cf[nt][3];
            }
        }
        __syncthreads();
        // trailing update of the lower tiles: A[r0.., r0..] -= P P^T
        {
            const int mt = R / 16;
            const int ntiles = mt * (mt + 1);  // sum over mi of (2 mi + 2)
            for (int tile = warp; tile < ntiles; tile += NWARPS)
            {
                // tile -> (mi, ni) with ni <= 2 mi + 1
                int mi = 0, base = 0;
                while (base + 2 * mi + 2 <= tile)
                {
                    base += 2 * mi + 2;
                    ++mi;
                }
                const int ni = tile - base;
                const int m0 = r0 + 16 * mi, n0 = r0 + 8 * ni;
                double *c = sa + (m0 + g) * PS + n0 + 2 * t;
                double cf[4] = { c[0], c[1], c[8 * PS], c[8 * PS + 1] };
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                {
                    double af[4], bf[2];
                    frag_a(af, sa, PS, m0, c0 + 8 * kk, g, t);
                    frag_bt(bf, sa, PS, n0, c0 + 8 * kk, g, t);
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                    {
                        af[e] = -af[e];
                    }
                    dmma(cf, af, bf);
                }
                c[0] = cf[0];
                c[1] = cf[1];
                c[8 * PS] = cf[2];
                c[8 * PS + 1] = cf[3];
            }
        }
        __syncthreads();
    }
    if (tid == 0 && bad != 0 && status != nullptr)
    {
        atomicCAS(&status->not_spd_row, 0, bad);
    }
    assemble_row_block(sa, xall + 3 * SB * XS, tbuf, 3, 0, NWARPS, 0);
    __syncthreads();
    pdl_launch_dependents();  // only the stores are left
    // store Linv (zero above the diagonal) in pairs of columns
#pragma unroll 8
    for (int q = 0; q < PB * PB / 2 / PTHREADS; ++q)
    {
        const int idx = q * PTHREADS + tid;
        const int i = idx >> 6, c = 2 * (idx & 63);
        if (i >= bs || c >= bs)
        {
            continue;
        }
        const double2 raw = *reinterpret_cast<const double2 *>(sa + i * PS + c);
        const double v0 = (c <= i) ? raw.x : 0.0;
        const double v1 = (c + 1 <= i) ? raw.y : 0.0;
        double *drow = (Linv != nullptr) ? Linv + static_cast<int64_t>(i) * ldi + c : nullptr;
        float *frow = (Linv32 != nullptr) ? Linv32 + static_cast<int64_t>(i) * ldi32 + c : nullptr;
        if (c + 1 < bs)
        {
            if (drow != nullptr)
            {
                *reinterpret_cast<double2 *>(drow) = make_double2(v0, v1);
            }
            if (frow != nullptr)
            {
                *reinterpret_cast<float2 *>(frow) = make_float2(static_cast<float>(v0), static_cast<float>(v1));
            }
        }
        else
        {
            if (drow != nullptr)
            {
                drow[0] = v0;
            }
            if (frow != nullptr)
            {
                frow[0] = static_cast<float>(v0);
            }
        }
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
    if ((ldi & 1) != 0 || (reinterpret_cast<uintptr_t>(Linv) & 15) != 0)
    {
        throw Error(1, "potrf_diag: Linv must be 16-byte aligned with an even leading dimension");
    }
    constexpr size_t smem = SMEM_DOUBLES * sizeof(double);
    ensure_smem_attr(reinterpret_cast<const void *>(potrf_inv_kernel<double>), static_cast<int>(smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(PTHREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1] = { programmatic_launch_attr() };
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    GPRAT_CUDA_CHECK(cudaLaunchKernelEx(&cfg, potrf_inv_kernel<double>, A, lda, bs, row0, Linv, ldi,
                                        static_cast<float *>(nullptr), int64_t{ 0 }, static_cast<double *>(nullptr),
                                        status, 1));
    GPRAT_LAUNCH_CHECK();
}

void potrf_diag_f32(float *A, int64_t lda, int bs, int row0, double *Linv, int64_t ldi, float *Linv32, int64_t ldi32,
                    double *diag, DeviceStatus *status, cudaStream_t s, bool write_l)
{
    if (bs <= 0 || bs > PB)
    {
        throw Error(1, "potrf_diag_f32: block size must be in [1, 128]");
    }
    if ((Linv != nullptr && ((ldi & 1) != 0 || (reinterpret_cast<uintptr_t>(Linv) & 15) != 0)) || (ldi32 & 1) != 0 ||
        (reinterpret_cast<uintptr_t>(Linv32) & 7) != 0)
    {
        throw Error(1, "potrf_diag_f32: Linv / Linv32 must be aligned with even leading dimensions");
    }
    constexpr size_t smem = SMEM_DOUBLES * sizeof(double);
    ensure_smem_attr(reinterpret_cast<const void *>(potrf_inv_kernel<float>), static_cast<int>(smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(PTHREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1] = { programmatic_launch_attr() };
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    GPRAT_CUDA_CHECK(
        cudaLaunchKernelEx(&cfg, potrf_inv_kernel<float>, A, lda, bs, row0, Linv, ldi, Linv32, ldi32, diag, status,
                           write_l ? 1 : 0));
    GPRAT_LAUNCH_CHECK();
}

}  // namespace gprat_cu
