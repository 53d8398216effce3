// FP64 tensor-core (DMMA, mma.sync m16n8k8 .f64) GEMM mainloop for sm_100a.
//
// Two CTA shapes share one mainloop (template parameter WN = warps along N):
//   WN = 4: CTA tile 128x128, 8 warps, 4-stage pipeline, 1 CTA/SM.  Used
//           when N <= 128 (panel solves, in-place diagonal-block steps).
//   WN = 2: CTA tile 128x64, 4 warps, 3-stage pipeline, 2 CTAs/SM, so one
//           CTA's C load/store overlaps the other CTA's DMMA main loop.
//           Used for the large trailing updates.
// Warp tile 64x32 = 4x4 m16n8k8 fragments (64 FP64 accumulators/thread).
// K step 16 via cp.async.  Shared-memory rows are padded so every fragment
// load is conflict-free (row stride = 4 mod 16 doubles when K is the
// contiguous index, 8 mod 16 when M/N is).  The epilogue is supplied by the
// kernel that instantiates the mainloop.
#pragma once

#include "common.cuh"

#include <type_traits>

namespace gprat_cu
{
namespace gemm
{

#ifndef GPRAT_DGEMM_BK
#define GPRAT_DGEMM_BK 16
#endif
constexpr int BK = GPRAT_DGEMM_BK;  // K per pipeline stage
constexpr int PAD_K = 4;  // stride BK+4 doubles (conflict-free fragment loads)
constexpr int PAD_T = 8;  // stride ROWS+8 doubles

template <int WN>
struct Cfg
{
    static constexpr int WM = 2;
    static constexpr int THREADS = 32 * WM * WN;
    static constexpr int BM = 64 * WM;  // 128
    static constexpr int BN = 32 * WN;  // 128 or 64
    static constexpr int STAGES = (WN == 4) ? (BK == 16 ? 4 : 3) : (BK == 16 ? 3 : 2);
    static constexpr int MIN_BLOCKS = (WN == 4) ? 1 : 2;
};

// Operand tile whose rows run along K: [ROWS][BK+PAD_K]
template <int ROWS>
struct KMajor
{
    static constexpr int SIZE = ROWS * (BK + PAD_K);
    __device__ __forceinline__ static int idx(int row, int k) { return row * (BK + PAD_K) + k; }
};

// Operand tile whose rows run along M or N: [BK][ROWS+PAD_T]
template <int ROWS>
struct RMajor
{
    static constexpr int SIZE = BK * (ROWS + PAD_T);
    __device__ __forceinline__ static int idx(int row, int k) { return k * (ROWS + PAD_T) + row; }
};

// A: transA=false -> A[m][k] rows along K -> KMajor; true -> RMajor.
// B: transB=true  -> B[n][k] rows along K -> KMajor; false -> RMajor.
template <bool TA, int ROWS>
using ALayout = typename std::conditional<TA, RMajor<ROWS>, KMajor<ROWS>>::type;
template <bool TB, int ROWS>
using BLayout = typename std::conditional<TB, KMajor<ROWS>, RMajor<ROWS>>::type;

template <int WN, bool TA, bool TB>
constexpr int smem_bytes()
{
    using C = Cfg<WN>;
    return C::STAGES * (ALayout<TA, C::BM>::SIZE + BLayout<TB, C::BN>::SIZE) * 8;
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

// Copies one operand tile (ROWS rows of the operand starting at r0, K range
// [k0, k0+BK)) into shared memory with zero fill outside [rows) x [K).
// KMAJOR: element (row, k) at P[row*ld + k]; otherwise at P[k*ld + row].
template <bool KMAJOR, int ROWS, int THREADS>
__device__ __forceinline__ void load_tile(double *s, const double *P, int64_t ld, int rows, int K, int r0, int k0,
                                          int tid)
{
    if (KMAJOR)
    {
        constexpr int CHUNKS = ROWS * (BK / 2);
#pragma unroll
        for (int i = 0; i < CHUNKS / THREADS; ++i)
        {
            int c = tid + i * THREADS;
            int row = c / (BK / 2);
            int kc = (c % (BK / 2)) * 2;
            int gr = r0 + row, gk = k0 + kc;
            int nv = (gr < rows) ? min(max(K - gk, 0), 2) : 0;
            const double *src = nv ? P + static_cast<int64_t>(gr) * ld + gk : P;
            cp_async16(s + KMajor<ROWS>::idx(row, kc), src, nv * 8);
        }
    }
    else
    {
        constexpr int PER_ROW = ROWS / 2;
        constexpr int CHUNKS = BK * PER_ROW;
#pragma unroll
        for (int i = 0; i < CHUNKS / THREADS; ++i)
        {
            int c = tid + i * THREADS;
            int krow = c / PER_ROW;
            int rc = (c % PER_ROW) * 2;
            int gk = k0 + krow, gr = r0 + rc;
            int nv = (gk < K) ? min(max(rows - gr, 0), 2) : 0;
            const double *src = nv ? P + static_cast<int64_t>(gk) * ld + gr : P;
            cp_async16(s + RMajor<ROWS>::idx(rc, krow), src, nv * 8);
        }
    }
}

struct TileCoord
{
    int m0, n0;
};

// Maps blockIdx to the C tile.  In `lower` mode the grid is 1-D over the
// tiles that touch the lower triangle: row tile i (BM high) has (i+1)*BM/BN
// column tiles.
template <int BM, int BN>
__device__ __forceinline__ TileCoord tile_coord(bool lower)
{
    TileCoord t;
    if (lower)
    {
        constexpr int R = BM / BN;
        const int q = blockIdx.x;
        int i = static_cast<int>((sqrt(8.0 * q / R + 1.0) - 1.0) * 0.5);
        while (R * (i + 1) * (i + 2) / 2 <= q)
        {
            ++i;
        }
        while (i > 0 && R * i * (i + 1) / 2 > q)
        {
            --i;
        }
        t.m0 = i * BM;
        t.n0 = (q - R * i * (i + 1) / 2) * BN;
    }
    else
    {
        t.m0 = blockIdx.y * BM;
        t.n0 = blockIdx.x * BN;
    }
    return t;
}

template <int BM, int BN>
inline int lower_grid(int M)
{
    const int t = (M + BM - 1) / BM;
    return (BM / BN) * t * (t + 1) / 2;
}

// acc[mi][ni][0..3]: rows wm*64+mi*16+g (+8 for [2],[3]), cols wn*32+ni*8+2t (+1)
struct Frag
{
    int g, t, wm, wn;
};

template <int WN>
__device__ __forceinline__ Frag frag_coords()
{
    Frag f;
    int lane = threadIdx.x & 31;
    int warp = threadIdx.x >> 5;
    f.g = lane >> 2;
    f.t = lane & 3;
    f.wm = warp / WN;  // 0..1
    f.wn = warp % WN;
    return f;
}

template <int WN, bool TA, bool TB>
__device__ __forceinline__ void mainloop(const GemmArgs &a, int m0, int n0, double *smem, double (&acc)[4][4][4],
                                         int k_begin, const Frag &f)
{
    using C = Cfg<WN>;
    using LA = ALayout<TA, C::BM>;
    using LB = BLayout<TB, C::BN>;
    constexpr int STAGES = C::STAGES;
    double *sA = smem;
    double *sB = smem + STAGES * LA::SIZE;
    const int tid = threadIdx.x;
    const int kspan = a.K - k_begin;
    const int KT = kspan > 0 ? (kspan + BK - 1) / BK : 0;

    auto load_stage = [&](int kt, int stage)
    {
        int k0 = k_begin + kt * BK;
        load_tile<!TA, C::BM, C::THREADS>(sA + stage * LA::SIZE, a.A, a.lda, a.M, a.K, m0, k0, tid);
        load_tile<TB, C::BN, C::THREADS>(sB + stage * LB::SIZE, a.B, a.ldb, a.N, a.K, n0, k0, tid);
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
                af[mi][0] = cA[LA::idx(r, c)];
                af[mi][1] = cA[LA::idx(r + 8, c)];
                af[mi][2] = cA[LA::idx(r, c + 4)];
                af[mi][3] = cA[LA::idx(r + 8, c + 4)];
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

}  // namespace gemm
}  // namespace gprat_cu
