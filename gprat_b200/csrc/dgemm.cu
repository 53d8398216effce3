// FP64 DMMA GEMM with the plain C-update epilogue (and optional fused
// row-sum-of-squares used by the variance solve).
//
// Uses in the pipeline (reference tile tasks they replace):
//   Cholesky trailing update  C -= P P^T, lower only  (syrk + gemm tasks,
//                              core/src/cpu/tiled_algorithms.cpp:33-55)
//   Cholesky panel solve      P = P Linv_kk^T, in place (trsm task, :21-32)
//   variance solve            W = W Linv_kk^T (+ rowsum W^2), W -= W_k L_k^T
//                              (forward_solve_tiled_matrix :117-149 with
//                              symmetric_matrix_matrix_diagonal_tiled :212-228)
#include "dgemm.cuh"

namespace gprat_cu
{
namespace
{

using namespace gemm;

template <int WN, bool TA, bool TB>
__global__ void __launch_bounds__(Cfg<WN>::THREADS, Cfg<WN>::MIN_BLOCKS) dgemm_kernel(GemmArgs a)
{
    using C = Cfg<WN>;
    extern __shared__ __align__(16) double smem[];
    const TileCoord tc = tile_coord<C::BM, C::BN>(a.lower);
    const int m0 = tc.m0, n0 = tc.n0;
    if (n0 >= a.N || m0 >= a.M)
    {
        return;
    }
    const Frag f = frag_coords<WN>();

    // Fused form (beta == 1, alpha == +-1): acc starts at alpha*C, the main
    // loop accumulates +A*B, and the store multiplies by alpha again, so
    // C_new = C + alpha*A*B without any per-fragment sign flips.
    const bool fused = (a.beta == 1.0) && (a.alpha == 1.0 || a.alpha == -1.0);
    const double osign = (fused && a.alpha == -1.0) ? -1.0 : 1.0;
    double acc[4][4][4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
    {
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
        {
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                int r = m0 + f.wm * 64 + mi * 16 + f.g + h * 8;
                int c = n0 + f.wn * 32 + ni * 8 + 2 * f.t;
                double v0 = 0.0, v1 = 0.0;
                if (fused && r < a.M)
                {
                    const double *cp = a.C + static_cast<int64_t>(r) * a.ldc + c;
                    if (c + 1 < a.N)
                    {
                        double2 v = *reinterpret_cast<const double2 *>(cp);
                        v0 = v.x;
                        v1 = v.y;
                    }
                    else if (c < a.N)
                    {
                        v0 = cp[0];
                    }
                }
                acc[mi][ni][2 * h] = osign * v0;
                acc[mi][ni][2 * h + 1] = osign * v1;
            }
        }
    }

    int k_begin = 0;
    if (a.k_tri > 0)
    {
        k_begin = (max(m0, n0) / BK) * BK;
    }
    mainloop<WN, TA, TB>(a, m0, n0, smem, acc, k_begin, f);

    // Epilogue: store (lower-only respected) and optional row sums of squares.
    double rs[4][2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
    {
        rs[mi][0] = 0.0;
        rs[mi][1] = 0.0;
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
    {
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
        {
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                int r = m0 + f.wm * 64 + mi * 16 + f.g + h * 8;
                int c = n0 + f.wn * 32 + ni * 8 + 2 * f.t;
                if (r >= a.M)
                {
                    continue;
                }
                double *cp = a.C + static_cast<int64_t>(r) * a.ldc + c;
                double v0 = osign * acc[mi][ni][2 * h], v1 = osign * acc[mi][ni][2 * h + 1];
                if (!fused)
                {
                    double o0 = 0.0, o1 = 0.0;
                    if (a.beta != 0.0)
                    {
                        if (c < a.N)
                        {
                            o0 = cp[0];
                        }
                        if (c + 1 < a.N)
                        {
                            o1 = cp[1];
                        }
                    }
                    v0 = a.alpha * v0 + a.beta * o0;
                    v1 = a.alpha * v1 + a.beta * o1;
                }
                bool w0 = c < a.N && (!a.lower || c <= r);
                bool w1 = c + 1 < a.N && (!a.lower || c + 1 <= r);
                if (w0 && w1)
                {
                    *reinterpret_cast<double2 *>(cp) = make_double2(v0, v1);
                }
                else
                {
                    if (w0)
                    {
                        cp[0] = v0;
                    }
                    if (w1)
                    {
                        cp[1] = v1;
                    }
                }
                rs[mi][h] += (w0 ? v0 * v0 : 0.0) + (w1 ? v1 * v1 : 0.0);
            }
        }
    }

    if (a.rowsq != nullptr)
    {
        // rows of this CTA: reduce over the quad (t), then over the N-warps.
        double *red = smem;  // [BM][WN], pipeline smem is free after mainloop
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
        {
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                double v = rs[mi][h];
                v += __shfl_xor_sync(0xffffffffu, v, 1);
                v += __shfl_xor_sync(0xffffffffu, v, 2);
                if (f.t == 0)
                {
                    red[(f.wm * 64 + mi * 16 + f.g + h * 8) * WN + f.wn] = v;
                }
            }
        }
        __syncthreads();
        for (int r = threadIdx.x; r < C::BM; r += C::THREADS)
        {
            int gr = m0 + r;
            if (gr < a.M)
            {
                double s = 0.0;
#pragma unroll
                for (int w = 0; w < WN; ++w)
                {
                    s += red[r * WN + w];
                }
                a.rowsq[gr] += s;
            }
        }
    }
}

template <int WN, bool TA, bool TB>
void launch(const GemmArgs &a, cudaStream_t s)
{
    using C = Cfg<WN>;
    constexpr int smem = smem_bytes<WN, TA, TB>();
    ensure_smem_attr(reinterpret_cast<const void *>(dgemm_kernel<WN, TA, TB>), smem);
    dim3 grid;
    if (a.lower)
    {
        grid = dim3(lower_grid<C::BM, C::BN>(a.M), 1, 1);
    }
    else
    {
        grid = dim3(ceil_div(a.N, C::BN), ceil_div(a.M, C::BM), 1);
    }
    const bool timed = gemm_timing_enabled();
    if (timed)
    {
        gemm_timing_begin(s);
    }
    dgemm_kernel<WN, TA, TB><<<grid, C::THREADS, smem, s>>>(a);
    GPRAT_LAUNCH_CHECK();
    if (timed)
    {
        const double mn = a.lower ? 0.5 * static_cast<double>(a.M) * (a.M + 1) : static_cast<double>(a.M) * a.N;
        gemm_timing_end(s, 2.0 * mn * a.K);
    }
}

template <int WN>
void dispatch(const GemmArgs &a, cudaStream_t s)
{
    if (a.transA)
    {
        a.transB ? launch<WN, true, true>(a, s) : launch<WN, true, false>(a, s);
    }
    else
    {
        a.transB ? launch<WN, false, true>(a, s) : launch<WN, false, false>(a, s);
    }
}

}  // namespace

void dgemm(const GemmArgs &a, cudaStream_t s)
{
    if (a.M <= 0 || a.N <= 0)
    {
        return;
    }
    if ((a.lda & 1) || (a.ldb & 1) || (a.ldc & 1) || (reinterpret_cast<uintptr_t>(a.A) & 15) ||
        (reinterpret_cast<uintptr_t>(a.B) & 15) || (reinterpret_cast<uintptr_t>(a.C) & 15))
    {
        throw Error(1, "dgemm: leading dimensions must be even and bases 16-byte aligned");
    }
    if (a.lower && a.M != a.N)
    {
        throw Error(1, "dgemm: lower mode needs M == N");
    }
    if (a.rowsq != nullptr && (a.N > 128 || a.lower))
    {
        throw Error(1, "dgemm: rowsq needs N <= 128 and full tiles");
    }
    // N <= 128: one CTA column covers every output column, which the in-place
    // panel solves and the fused row sums rely on.  Wider problems use the
    // 2-CTA/SM shape.
    if (a.N <= 128)
    {
        dispatch<4>(a, s);
    }
    else
    {
        dispatch<2>(a, s);
    }
}

}  // namespace gprat_cu
