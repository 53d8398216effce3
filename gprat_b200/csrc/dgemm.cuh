// FP64 tensor-core (DMMA, mma.sync m16n8k8 .f64) GEMM mainloop for sm_100a.
//
// CTA tile 128x128, K step 16, 4-stage cp.async pipeline, 8 warps laid out
// 2 (M) x 4 (N), warp tile 64x32 = 4x4 m16n8k8 fragments.  Shared-memory
// rows are padded so that every fragment load is conflict-free (row stride
// = 4 mod 16 doubles when K is the contiguous index, 8 mod 16 when M/N is).
// The epilogue is a template parameter: plain C update (dgemm.cu) or the
// fused adjoint trace (optimizer.cu).
#pragma once

#include "common.cuh"

namespace gprat_cu
{
namespace gemm
{

constexpr int BM = 128;
constexpr int BN = 128;
constexpr int BK = 16;
constexpr int STAGES = 4;
constexpr int THREADS = 256;
constexpr int PAD_K = 4;  // stride BK+4 = 20 doubles
constexpr int PAD_T = 8;  // stride BM+8 = 136 doubles

template <bool T>
struct OpLayout;  // operand whose rows run along K (T=false for A, true for B)

// "K-contiguous" operand tile: [rows][BK+PAD_K]
struct KMajor
{
    static constexpr int SIZE = BM * (BK + PAD_K);
    __device__ __forceinline__ static int idx(int row, int k) { return row * (BK + PAD_K) + k; }
};

// "row-contiguous" operand tile: [BK][rows+PAD_T]
struct RMajor
{
    static constexpr int SIZE = BK * (BM + PAD_T);
    __device__ __forceinline__ static int idx(int row, int k) { return k * (BM + PAD_T) + row; }
};

// A: transA=false -> A[m][k] rows along K -> KMajor; true -> RMajor.
// B: transB=true  -> B[n][k] rows along K -> KMajor; false -> RMajor.
template <bool TA>
using ALayout = typename std::conditional<TA, RMajor, KMajor>::type;
template <bool TB>
using BLayout = typename std::conditional<TB, KMajor, RMajor>::type;

template <bool TA, bool TB>
constexpr int smem_bytes()
{
    return STAGES * (ALayout<TA>::SIZE + BLayout<TB>::SIZE) * 8;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes)
{
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Copies one operand tile (rows [r0, r0+128) of the operand, K range
// [k0, k0+16)) into shared memory.  `trans` selects the global layout:
// false -> element (row, k) at P[row*ld + k]; true -> at P[k*ld + row].
template <bool KMAJOR>
__device__ __forceinline__ void load_tile(double *s, const double *P, int64_t ld, int rows, int K, int r0, int k0,
                                          int tid)
{
    if (KMAJOR)
    {
        // 128 rows x 8 chunks of 2 doubles
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            int c = tid + i * THREADS;
            int row = c >> 3;
            int kc = (c & 7) * 2;
            int gr = r0 + row, gk = k0 + kc;
            int nv = (gr < rows) ? min(max(K - gk, 0), 2) : 0;
            const double *src = nv ? P + static_cast<int64_t>(gr) * ld + gk : P;
            cp_async16(s + KMajor::idx(row, kc), src, nv * 8);
        }
    }
    else
    {
        // 16 k-rows x 64 chunks of 2 doubles
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            int c = tid + i * THREADS;
            int krow = c >> 6;
            int rc = (c & 63) * 2;
            int gk = k0 + krow, gr = r0 + rc;
            int nv = (gk < K) ? min(max(rows - gr, 0), 2) : 0;
            const double *src = nv ? P + static_cast<int64_t>(gk) * ld + gr : P;
            cp_async16(s + RMajor::idx(rc, krow), src, nv * 8);
        }
    }
}

struct TileCoord
{
    int m0, n0;
    bool skip;
};

// Maps blockIdx to the C tile; in `lower` mode the grid is 1-D over the
// lower-triangular tiles (j <= i).
__device__ __forceinline__ TileCoord tile_coord(bool lower)
{
    TileCoord t;
    t.skip = false;
    if (lower)
    {
        int q = blockIdx.x;
        int i = static_cast<int>((sqrt(8.0 * q + 1.0) - 1.0) * 0.5);
        while ((i + 1) * (i + 2) / 2 <= q)
        {
            ++i;
        }
        while (i * (i + 1) / 2 > q)
        {
            --i;
        }
        int j = q - i * (i + 1) / 2;
        t.m0 = i * BM;
        t.n0 = j * BN;
    }
    else
    {
        t.m0 = blockIdx.y * BM;
        t.n0 = blockIdx.x * BN;
    }
    return t;
}

// acc[mi][ni][0..3]: rows wm*64+mi*16+g (+8 for [2],[3]), cols wn*32+ni*8+2t (+1)
struct Frag
{
    int g, t, wm, wn;
};

template <bool TA, bool TB>
__device__ __forceinline__ void mainloop(const GemmArgs &a, int m0, int n0, double *smem, double (&acc)[4][4][4],
                                         bool negate, int k_begin, const Frag &f)
{
    using LA = ALayout<TA>;
    using LB = BLayout<TB>;
    double *sA = smem;
    double *sB = smem + STAGES * LA::SIZE;
    const int tid = threadIdx.x;
    const int kspan = a.K - k_begin;
    const int KT = kspan > 0 ? (kspan + BK - 1) / BK : 0;

    auto load_stage = [&](int kt, int stage)
    {
        int k0 = k_begin + kt * BK;
        // A tile: rows = M dimension
        load_tile<!TA>(sA + stage * LA::SIZE, a.A, a.lda, a.M, a.K, m0, k0, tid);
        // B tile: rows = N dimension
        load_tile<TB>(sB + stage * LB::SIZE, a.B, a.ldb, a.N, a.K, n0, k0, tid);
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s)
    {
        if (s < KT)
        {
            load_stage(s, s);
        }
        cp_async_commit();
    }

    const double sgn = negate ? -1.0 : 1.0;
    for (int kt = 0; kt < KT; ++kt)
    {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        int nk = kt + STAGES - 1;
        if (nk < KT)
        {
            load_stage(nk, nk % STAGES);
        }
        cp_async_commit();

        const double *cA = sA + (kt % STAGES) * LA::SIZE;
        const double *cB = sB + (kt % STAGES) * LB::SIZE;
#pragma unroll
        for (int ks = 0; ks < BK / 8; ++ks)
        {
            double af[4][4];
            double bf[4][2];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
            {
                int r = f.wm * 64 + mi * 16 + f.g;
                int c = ks * 8 + f.t;
                af[mi][0] = sgn * cA[LA::idx(r, c)];
                af[mi][1] = sgn * cA[LA::idx(r + 8, c)];
                af[mi][2] = sgn * cA[LA::idx(r, c + 4)];
                af[mi][3] = sgn * cA[LA::idx(r + 8, c + 4)];
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
            {
                int n = f.wn * 32 + ni * 8 + f.g;
                int k = ks * 8 + f.t;
                bf[ni][0] = cB[LB::idx(n, k)];
                bf[ni][1] = cB[LB::idx(n, k + 4)];
            }
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
            {
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                {
                    dmma_16x8x8(acc[mi][ni], af[mi], bf[ni]);
                }
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();
}

__device__ __forceinline__ Frag frag_coords()
{
    Frag f;
    int lane = threadIdx.x & 31;
    int warp = threadIdx.x >> 5;
    f.g = lane >> 2;
    f.t = lane & 3;
    f.wm = warp >> 2;  // 0..1
    f.wn = warp & 3;   // 0..3
    return f;
}

}  // namespace gemm
}  // namespace gprat_cu
