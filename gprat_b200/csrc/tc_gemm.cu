// tcgen05 tensor-core GEMM for the mixed-precision path (sm_100a).
//
//   C[MxN] (FP32, row-major) = beta*C + alpha * A B^T
//   A (M x K), B (N x K): K-contiguous FP32 (kind::tf32) or BF16 (kind::f16)
//
// Persistent, warp-specialised CTA (320 threads, one CTA per SM):
//   warp 0, one lane : TMA producer -- 128x128-byte tiles of A and B per
//                      stage (128-byte swizzle), 7-stage ring, mbarrier
//                      complete_tx accounting; no multicast;
//   warp 1, one lane : MMA issuer -- 4 x tcgen05.mma (M=128, N=128) per
//                      stage into a TMEM accumulator, tcgen05.commit frees the
//                      smem stage; two accumulators (256 TMEM columns) so the
//                      epilogue of tile i overlaps the MMAs of tile i+1;
//   warps 2..9       : epilogue -- two warps per TMEM lane quarter, 64 columns
//                      each: tcgen05.ld of the accumulator, release it, scale
//                      (and mask above the diagonal), stage each 32 x 32
//                      sub-tile in shared memory in the TMA box layout, then
//                      one TMA bulk tensor store (beta = 0) or reduce-add
//                      (beta = 1) per sub-tile: C is never read by the SM, and
//                      its rows are written as whole 128-byte lines
//                      (optional FP64 row sums of squares, beta = 0 only).
// Every mbarrier wait is bounded (about 2 s of device time); a wait that gives
// up raises a CTA-wide abort flag, the roles leave their loops, in-flight
// TMA copies are given time to land, the MMA issuer drains its own MMAs, the
// TMEM is freed and the status word's timeout flag is set.
#include "tc_gemm.cuh"
#include "tcgen05_ptx.cuh"

#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

namespace gprat_cu
{
namespace
{

using namespace tcx;

constexpr int TM = 128;
constexpr int TN = 128;                // N of the narrow tile (row sums of squares need N <= TN)
constexpr int TILE_BYTES = 128 * 128;  // one 128-row x 128-byte operand tile (one TMA box)
constexpr int NUM_THREADS = 320;  // warp 0 TMA, warp 1 MMA, warps 2..9 epilogue
constexpr int EPI_WARPS = 8;
constexpr int EPI_BUF_BYTES = 32 * 128;  // one 32 x 32 FP32 sub-tile (TMA box, 128-byte swizzle)

// Tile shape: 128 x TNV (TNV = 128 or 256).  The wide tile halves the A
// traffic per flop and lowers the shared-memory bandwidth the MMA and the
// TMA fills need (operand reads + fills per flop: 3/4 of the narrow tile's).
template <int TNV>
struct TileCfg
{
    static constexpr int STAGE_BYTES = TILE_BYTES + (TNV / 128) * TILE_BYTES;  // A + B
    static constexpr int STAGES = (TNV == 128) ? 6 : 4;
    static constexpr int TMEM_COLS = 2 * TNV;  // two accumulators
    static constexpr int EPI_COLS = TNV / 2;   // columns per epilogue warp
    static constexpr int SMEM_BYTES = 1024 + STAGES * STAGE_BYTES + EPI_WARPS * EPI_BUF_BYTES + 256;
};

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, const void *src, int x, int y)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(smem_u32(src)), "r"(x), "r"(y)
                 : "memory");
}

__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap *map, const void *src, int x, int y)
{
    asm volatile("cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(smem_u32(src)), "r"(x), "r"(y)
                 : "memory");
}

// Instruction descriptor: D = F32, A/B format (1 = BF16, 2 = TF32), both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t make_idesc(uint32_t fmt, int n)
{
    return (1u << 4) | (fmt << 7) | (fmt << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(TM >> 4) << 24);
}

template <int KIND>
__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    if (KIND == static_cast<int>(TcKind::TF32))
    {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
    }
    else
    {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
    }
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int j = 0; j < 32; ++j)
    {
        v[j] = __uint_as_float(r[j]);
    }
}


// Full (non-lower) tile index t -> (row tile, column tile) in groups of
// GROUP_M row tiles: a group sweeps its columns together, so the tiles in
// flight at one time (one per CTA or CTA pair) share a few row panels of A
// and a few column panels of B.  For deep updates (K in the thousands) an
// operand panel is tens of MB and the L2 cannot keep one panel per tile in
// flight; the grouping then cuts the HBM re-reads of B by about GROUP_M.
constexpr int GROUP_M = 8;

__device__ __forceinline__ void grouped_tile(int t, int tiles_n, int ntiles, int &tm, int &tn)
{
    const int tiles_m = ntiles / tiles_n;
    const int span = GROUP_M * tiles_n;
    const int g = t / span;
    const int first = g * GROUP_M;
    const int gm = min(tiles_m - first, GROUP_M);
    const int r = t - g * span;
    tm = first + r % gm;
    tn = r / gm;
}

// Tile t -> (m0, n0).  Lower mode (M == N): row tile i holds the column
// tiles that reach the diagonal or below, (i * TM) / TNV + 1 of them.
template <int TNV>
__device__ __forceinline__ void tile_of(int t, bool lower, int tiles_n, int ntiles, int &m0, int &n0)
{
    if (!lower)
    {
        int tm, tn;
        grouped_tile(t, tiles_n, ntiles, tm, tn);
        m0 = tm * TM;
        n0 = tn * TNV;
        return;
    }
    if (TNV == TM)
    {
        // prefix(i) = i (i + 1) / 2
        int i = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
        while ((i + 1) * (i + 2) / 2 <= t)
        {
            ++i;
        }
        while (i > 0 && i * (i + 1) / 2 > t)
        {
            --i;
        }
        m0 = i * TM;
        n0 = (t - i * (i + 1) / 2) * TNV;
    }
    else
    {
        // TNV = 2 TM: row tile i holds i / 2 + 1 column tiles;
        // prefix(2a) = a (a + 1), prefix(2a + 1) = (a + 1)^2
        auto prefix = [](int i)
        {
            const int a = i >> 1;
            return (i & 1) ? (a + 1) * (a + 1) : a * (a + 1);
        };
        int i = static_cast<int>(2.0 * sqrt(static_cast<double>(t))) - 2;
        i = i < 0 ? 0 : i;
        while (prefix(i + 1) <= t)
        {
            ++i;
        }
        while (i > 0 && prefix(i) > t)
        {
            --i;
        }
        m0 = i * TM;
        n0 = (t - prefix(i)) * TNV;
    }
}

template <int KIND, int TNV>
__global__ void __launch_bounds__(NUM_THREADS, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const __grid_constant__ CUtensorMap tmC, TcGemmArgs p, int tiles_n, int ntiles)
{
    using Cfg = TileCfg<TNV>;
    constexpr int STAGES = Cfg::STAGES;
    constexpr int STAGE_BYTES = Cfg::STAGE_BYTES;
    constexpr int EPI_COLS = Cfg::EPI_COLS;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *tiles = smem;
    uint8_t *epi_smem = smem + STAGES * STAGE_BYTES;  // 1024-byte aligned sub-tile buffers
    uint64_t *full = reinterpret_cast<uint64_t *>(epi_smem + EPI_WARPS * EPI_BUF_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *drain = tempty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    constexpr int KSTAGE = (KIND == static_cast<int>(TcKind::TF32)) ? 32 : 64;  // elements per 128 bytes
    constexpr uint32_t IDESC = make_idesc(KIND == static_cast<int>(TcKind::TF32) ? 2u : 1u, TNV);
    const int kiters = p.K / KSTAGE;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < STAGES; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b)
        {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 256);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(Cfg::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    pdl_wait();  // the previous kernel's results are visible from here on

    if (warp == 0)
    {
        if (lane == 0)
        {
            // ---------------- TMA producer ----------------
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            for (int t = blockIdx.x; ok && t < ntiles; t += gridDim.x)
            {
                int m0, n0;
                tile_of<TNV>(t, p.lower, tiles_n, ntiles, m0, n0);
                for (int k = 0; k < kiters; ++k)
                {
                    if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag))
                    {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full[s], STAGE_BYTES);
                    uint8_t *st = tiles + s * STAGE_BYTES;
                    tma_load_2d(st, &tmA, &full[s], p.a_col0 + k * KSTAGE, p.a_row0 + m0);
#pragma unroll
                    for (int bh = 0; bh < TNV / 128; ++bh)
                    {
                        tma_load_2d(st + TILE_BYTES * (1 + bh), &tmB, &full[s], p.b_col0 + k * KSTAGE,
                                    p.b_row0 + n0 + 128 * bh);
                    }
                    if (++s == STAGES)
                    {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (*abort_flag)
            {
                // give copies already in flight time to land before the CTA exits
                const unsigned long long t0 = global_ns();
                while (global_ns() - t0 < 200000ull)
                {
                }
            }
        }
    }
    else if (warp == 1)
    {
        if (lane == 0)
        {
            // ---------------- MMA issuer ----------------
            int s = 0;
            uint32_t ph = 0;
            uint32_t acc_bits = 0u;
            bool ok = true;
            int it = 0;
            for (int t = blockIdx.x; ok && t < ntiles; t += gridDim.x, ++it)
            {
                const int b = it & 1;
                if (!mbar_wait(&tempty[b], ((acc_bits >> b) & 1u) ^ 1u, abort_flag))
                {
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem_base + static_cast<uint32_t>(b * TNV);
                for (int k = 0; k < kiters; ++k)
                {
                    if (!mbar_wait(&full[s], ph, abort_flag))
                    {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(tiles + s * STAGE_BYTES);
                    const uint64_t adesc = sw128_desc(a_addr);
                    const uint64_t bdesc = sw128_desc(a_addr + TILE_BYTES);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                    {
                        // 32 bytes of K per instruction: advance the start address by 2 x 16 B
                        mma_issue<KIND>(d, adesc + 2 * kk, bdesc + 2 * kk, IDESC, (k | kk) != 0 ? 1u : 0u);
                    }
                    mma_commit(&empty[s]);
                    if (++s == STAGES)
                    {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok)
                {
                    break;
                }
                mma_commit(&tfull[b]);
                acc_bits ^= 1u << b;
            }
            // drain: arrives once every MMA issued above has completed
            mma_commit(drain);
            mbar_wait(drain, 0u, abort_flag);
        }
    }
    else
    {
        // ---------------- epilogue (warps 2..9) ----------------
        // two warps per TMEM lane quarter, each owning half of the TNV columns,
        // read from TMEM and written out 32 columns at a time
        const int ew = warp - 2;
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        const int h = ew >> 2;   // column half
        const int r_in = q * 32 + lane;
        uint8_t *buf = epi_smem + ew * EPI_BUF_BYTES;
        const uint32_t buf_row = smem_u32(buf) + static_cast<uint32_t>(lane) * 128u;
        uint32_t acc_bits = 0u;  // phase bit of each accumulator
        int it = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it)
        {
            const int b = it & 1;
            int m0, n0;
            tile_of<TNV>(t, p.lower, tiles_n, ntiles, m0, n0);
            if (!mbar_wait(&tfull[b], (acc_bits >> b) & 1u, abort_flag))
            {
                break;
            }
            tc_fence_after();
            const uint32_t taddr = tmem_base + (static_cast<uint32_t>(q * 32) << 16) +
                                   static_cast<uint32_t>(b * TNV + h * EPI_COLS);
            const int row = m0 + r_in;
            const int row0 = m0 + q * 32;  // first row of this warp's sub-tiles
            const bool diag = p.lower && n0 + TNV > m0;  // tile reaches above the diagonal
            double sq = 0.0;
            // the whole accumulator slice into registers first, then release it
            // to the MMA warp before any shared-memory or TMA work
            float v[EPI_COLS];
#pragma unroll
            for (int c = 0; c < EPI_COLS / 32; ++c)
            {
                tmem_ld32(taddr + c * 32, v + c * 32);
            }
            tmem_ld_wait();
            tc_fence_before();
            mbar_arrive(&tempty[b]);
#pragma unroll
            for (int c = 0; c < EPI_COLS / 32; ++c)
            {
                const int col0 = n0 + h * EPI_COLS + c * 32;
                // warp-uniform: sub-tile outside C, or entirely above the diagonal
                if (col0 >= p.N || (diag && col0 >= row0 + 32))
                {
                    continue;
                }
                float w[32];
#pragma unroll
                for (int j = 0; j < 32; ++j)
                {
                    float val = p.alpha * v[c * 32 + j];
                    if (diag && col0 + j > row)
                    {
                        val = 0.0f;
                    }
                    w[j] = val;
                    if (p.rowsq != nullptr && col0 + j < p.N)
                    {
                        sq += static_cast<double>(val) * val;
                    }
                }
                // the previous bulk operation of this warp must have read the buffer
                if (lane == 0)
                {
                    bulk_wait_read_all();
                }
                __syncwarp();
#pragma unroll
                for (int j = 0; j < 8; ++j)
                {
                    const uint32_t addr = buf_row + (static_cast<uint32_t>(j ^ (lane & 7)) << 4);
                    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(w[4 * j]),
                                 "f"(w[4 * j + 1]), "f"(w[4 * j + 2]), "f"(w[4 * j + 3])
                                 : "memory");
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0)
                {
                    if (p.beta != 0.0f)
                    {
                        tma_reduce_add_2d(&tmC, buf, col0, row0);
                    }
                    else
                    {
                        tma_store_2d(&tmC, buf, col0, row0);
                    }
                    bulk_commit();
                }
            }
            acc_bits ^= 1u << b;
            if (p.rowsq != nullptr && row < p.M)
            {
                p.rowsq[h * p.rowsq_half + row] += sq;  // single writer per word and launch
            }
        }
        // the CTA's last tile is in its stores: the next kernel in the stream
        // may start its set-up (its CTAs then wait on free SMs, so the
        // signal comes late enough not to hold SMs other streams could use)
        pdl_launch_dependents();
        if (lane == 0)
        {
            bulk_wait_all();
        }
        __syncwarp();
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(Cfg::TMEM_COLS));
    }
    if (threadIdx.x == 0 && *abort_flag && p.status != nullptr)
    {
        atomicExch(&p.status->timeout, 1);
    }
}

// ---------------------------------------------------------------------------
// CTA-pair variant: a cluster of two CTAs computes one 256 x 256 tile with
// tcgen05.mma.cta_group::2 (M = 256 across the pair, N = 256).  Each CTA loads
// its own 128 rows of A and its own 128 rows of B (plain TMA loads, no
// multicast; the transaction bytes of both CTAs complete the leader's stage
// barrier); the leader's single MMA thread reads A from each CTA's shared
// memory for that CTA's rows and B from both, and accumulates each CTA's 128 x
// 256 half in that CTA's TMEM.  Per SM this moves 32 KB of operands per
// 128 x 256 x 32 step instead of 48 KB for the single-CTA 128 x 256 tile.
//   leader (rank 0): TMA warp (its halves + expect_tx for both), MMA warp,
//                    8 epilogue warps for rows m0 .. m0+127
//   peer   (rank 1): TMA warp (its halves), 8 epilogue warps for rows m0+128 ..
// Stage barriers: full[s] (leader; both CTAs' TMA bytes), empty[s] (both;
// the leader's commit arrives on both), tfull[b] (both; multicast commit),
// tempty[b] (leader; one arrival per epilogue warp of either CTA).
constexpr int PAIR_STAGE_BYTES = 2 * TILE_BYTES;  // per CTA: A half + B half
constexpr int PAIR_STAGES = 6;
constexpr int PAIR_TN = 256;
constexpr int PAIR_TMEM_COLS = 2 * PAIR_TN;
constexpr int PAIR_SMEM_BYTES = 1024 + PAIR_STAGES * PAIR_STAGE_BYTES + EPI_WARPS * EPI_BUF_BYTES + 256;

__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *map, uint32_t leader_bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(leader_bar), "r"(x), "r"(y)
        : "memory");
}

template <int KIND>
__device__ __forceinline__ void mma_issue_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                               uint32_t accumulate)
{
    if (KIND == static_cast<int>(TcKind::TF32))
    {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
    }
    else
    {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
    }
}

// pair tile t -> (m0, n0) in units of 256 (lower: square tiles at or below the diagonal)
__device__ __forceinline__ void pair_tile_of(int t, bool lower, int tiles_n, int ntiles, int &m0, int &n0)
{
    if (!lower)
    {
        int tm, tn;
        grouped_tile(t, tiles_n, ntiles, tm, tn);
        m0 = tm * 256;
        n0 = tn * 256;
        return;
    }
    int i = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= t)
    {
        ++i;
    }
    while (i > 0 && i * (i + 1) / 2 > t)
    {
        --i;
    }
    m0 = i * 256;
    n0 = (t - i * (i + 1) / 2) * 256;
}

template <int KIND>
__global__ void __launch_bounds__(NUM_THREADS, 1)
    tc_gemm_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                        const __grid_constant__ CUtensorMap tmC, TcGemmArgs p, int tiles_n, int ntiles)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *tiles = smem;
    uint8_t *epi_smem = smem + PAIR_STAGES * PAIR_STAGE_BYTES;
    uint64_t *full = reinterpret_cast<uint64_t *>(epi_smem + EPI_WARPS * EPI_BUF_BYTES);
    uint64_t *empty = full + PAIR_STAGES;
    uint64_t *tfull = empty + PAIR_STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *drain = tempty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1;
    const int npairs = gridDim.x >> 1;
    constexpr int KSTAGE = (KIND == static_cast<int>(TcKind::TF32)) ? 32 : 64;
    constexpr uint32_t IDESC = (1u << 4) | ((KIND == static_cast<int>(TcKind::TF32) ? 2u : 1u) << 7) |
                               ((KIND == static_cast<int>(TcKind::TF32) ? 2u : 1u) << 10) |
                               (static_cast<uint32_t>(PAIR_TN >> 3) << 17) | (static_cast<uint32_t>(256 >> 4) << 24);
    const int kiters = p.K / KSTAGE;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < PAIR_STAGES; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b)
        {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 2 * EPI_WARPS);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(PAIR_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::);
    }
    tc_fence_before();
    cluster_sync_all();  // barriers of both CTAs initialised, TMEM allocated
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    pdl_wait();  // the previous kernel's results are visible from here on

    if (warp == 0)
    {
        if (lane == 0)
        {
            // ---------------- TMA producer (both CTAs) ----------------
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            for (int t = pair; ok && t < ntiles; t += npairs)
            {
                int m0, n0;
                pair_tile_of(t, p.lower, tiles_n, ntiles, m0, n0);
                const int arow = p.a_row0 + m0 + 128 * static_cast<int>(rank);
                const int brow = p.b_row0 + n0 + 128 * static_cast<int>(rank);
                for (int k = 0; k < kiters; ++k)
                {
                    if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag))
                    {
                        ok = false;
                        break;
                    }
                    if (leader)
                    {
                        mbar_expect_tx(&full[s], 2 * PAIR_STAGE_BYTES);  // both CTAs' bytes
                    }
                    const uint32_t bar = map_to_rank(&full[s], 0);
                    uint8_t *st = tiles + s * PAIR_STAGE_BYTES;
                    tma_load_2d_pair(st, &tmA, bar, p.a_col0 + k * KSTAGE, arow);
                    tma_load_2d_pair(st + TILE_BYTES, &tmB, bar, p.b_col0 + k * KSTAGE, brow);
                    if (++s == PAIR_STAGES)
                    {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (*abort_flag)
            {
                const unsigned long long t0 = global_ns();
                while (global_ns() - t0 < 200000ull)
                {
                }
            }
        }
    }
    else if (warp == 1)
    {
        if (lane == 0 && leader)
        {
            // ---------------- MMA issuer (leader only) ----------------
            int s = 0;
            uint32_t ph = 0;
            uint32_t acc_bits = 0u;
            bool ok = true;
            int it = 0;
            for (int t = pair; ok && t < ntiles; t += npairs, ++it)
            {
                const int b = it & 1;
                if (!mbar_wait(&tempty[b], ((acc_bits >> b) & 1u) ^ 1u, abort_flag))
                {
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem_base + static_cast<uint32_t>(b * PAIR_TN);
                for (int k = 0; k < kiters; ++k)
                {
                    if (!mbar_wait(&full[s], ph, abort_flag))
                    {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(tiles + s * PAIR_STAGE_BYTES);
                    const uint64_t adesc = sw128_desc(a_addr);
                    const uint64_t bdesc = sw128_desc(a_addr + TILE_BYTES);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                    {
                        mma_issue_pair<KIND>(d, adesc + 2 * kk, bdesc + 2 * kk, IDESC, (k | kk) != 0 ? 1u : 0u);
                    }
                    mma_commit_pair_both(&empty[s]);
                    if (++s == PAIR_STAGES)
                    {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok)
                {
                    break;
                }
                mma_commit_pair_both(&tfull[b]);
                acc_bits ^= 1u << b;
            }
            mma_commit_pair_local(drain);
            mbar_wait(drain, 0u, abort_flag);
        }
    }
    else
    {
        // ---------------- epilogue (warps 2..9 of both CTAs) ----------------
        constexpr int EPI_COLS = PAIR_TN / 2;
        const int ew = warp - 2;
        const int q = warp & 3;
        const int h = ew >> 2;
        uint8_t *buf = epi_smem + ew * EPI_BUF_BYTES;
        const uint32_t buf_row = smem_u32(buf) + static_cast<uint32_t>(lane) * 128u;
        uint32_t acc_bits = 0u;
        int it = 0;
        for (int t = pair; t < ntiles; t += npairs, ++it)
        {
            const int b = it & 1;
            int mp, n0;
            pair_tile_of(t, p.lower, tiles_n, ntiles, mp, n0);
            const int m0 = mp + 128 * static_cast<int>(rank);  // this CTA's rows
            if (!mbar_wait(&tfull[b], (acc_bits >> b) & 1u, abort_flag))
            {
                break;
            }
            tc_fence_after();
            const uint32_t taddr = tmem_base + (static_cast<uint32_t>(q * 32) << 16) +
                                   static_cast<uint32_t>(b * PAIR_TN + h * EPI_COLS);
            float v[EPI_COLS];
#pragma unroll
            for (int c = 0; c < EPI_COLS / 32; ++c)
            {
                tmem_ld32(taddr + c * 32, v + c * 32);
            }
            tmem_ld_wait();
            tc_fence_before();
            __syncwarp();
            if (lane == 0)
            {
                mbar_arrive_cluster(map_to_rank(&tempty[b], 0));
            }
            acc_bits ^= 1u << b;
            const int row = m0 + q * 32 + lane;
            const int row0 = m0 + q * 32;
            const bool diag = p.lower && n0 + PAIR_TN > m0;
#pragma unroll
            for (int c = 0; c < EPI_COLS / 32; ++c)
            {
                const int col0 = n0 + h * EPI_COLS + c * 32;
                if (col0 >= p.N || row0 >= p.M || (diag && col0 >= row0 + 32))
                {
                    continue;
                }
                float w[32];
#pragma unroll
                for (int j = 0; j < 32; ++j)
                {
                    float val = p.alpha * v[c * 32 + j];
                    if (diag && col0 + j > row)
                    {
                        val = 0.0f;
                    }
                    w[j] = val;
                }
                if (lane == 0)
                {
                    bulk_wait_read_all();
                }
                __syncwarp();
#pragma unroll
                for (int j = 0; j < 8; ++j)
                {
                    const uint32_t addr = buf_row + (static_cast<uint32_t>(j ^ (lane & 7)) << 4);
                    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(w[4 * j]),
                                 "f"(w[4 * j + 1]), "f"(w[4 * j + 2]), "f"(w[4 * j + 3])
                                 : "memory");
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0)
                {
                    if (p.beta != 0.0f)
                    {
                        tma_reduce_add_2d(&tmC, buf, col0, row0);
                    }
                    else
                    {
                        tma_store_2d(&tmC, buf, col0, row0);
                    }
                    bulk_commit();
                }
            }
        }
        // the CTA's last tile is in its stores: the next kernel in the stream
        // may start its set-up (its CTAs then wait on free SMs, so the
        // signal comes late enough not to hold SMs other streams could use)
        pdl_launch_dependents();
        if (lane == 0)
        {
            bulk_wait_all();
        }
        __syncwarp();
    }

    tc_fence_before();
    cluster_sync_all();  // no CTA leaves while its peer may still signal or read it
    if (warp == 0)
    {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(PAIR_TMEM_COLS));
    }
    if (threadIdx.x == 0 && *abort_flag && p.status != nullptr)
    {
        atomicExch(&p.status->timeout, 1);
    }
}

template <typename T>
__global__ void convert_kernel(const T *__restrict__ src, int64_t lds, void *__restrict__ dst, int64_t ldd, int rows,
                               int cols, int mode)
{
    const int64_t total = static_cast<int64_t>(rows) * cols;
    for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < total;
         q += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const int64_t r = q / cols, c = q % cols;
        const T v = src[r * lds + c];
        if (mode == 0)
        {
            static_cast<float *>(dst)[r * ldd + c] = static_cast<float>(v);
        }
        else if (mode == 1)
        {
            static_cast<double *>(dst)[r * ldd + c] = static_cast<double>(v);
        }
        else
        {
            static_cast<__nv_bfloat16 *>(dst)[r * ldd + c] = __float2bfloat16_rn(static_cast<float>(v));
        }
    }
}

template <typename T>
void launch_convert(const T *src, int64_t lds, void *dst, int64_t ldd, int rows, int cols, int mode, cudaStream_t s)
{
    if (rows <= 0 || cols <= 0)
    {
        return;
    }
    const int64_t total = static_cast<int64_t>(rows) * cols;
    const int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, 148 * 16));
    convert_kernel<T><<<blocks, 256, 0, s>>>(src, lds, dst, ldd, rows, cols, mode);
    GPRAT_LAUNCH_CHECK();
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once,
                   []
                   {
                       void *p = nullptr;
                       cudaDriverEntryPointQueryResult q;
                       if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                                            &q) == cudaSuccess &&
                           q == cudaDriverEntryPointSuccess)
                       {
                           fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
                       }
                   });
    if (fn == nullptr)
    {
        throw Error(4, "cuTensorMapEncodeTiled is not available from the driver");
    }
    return fn;
}

int sm_count() { return device_sm_count(); }

}  // namespace

int device_sm_count()
{
    int dev = 0, n = 0;
    GPRAT_CUDA_CHECK(cudaGetDevice(&dev));
    GPRAT_CUDA_CHECK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

void tc_make_operand(TcOperand &op, const void *base, int rows, int cols, int64_t ld, TcKind kind)
{
    const int esize = (kind == TcKind::TF32) ? 4 : 2;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || ((ld * esize) & 15) || rows <= 0 || cols <= 0)
    {
        throw Error(1, "tc_make_operand: base must be 16-byte aligned and ld * element size a multiple of 16");
    }
    op.base = base;
    op.rows = rows;
    op.cols = cols;
    op.ld = ld;
    op.kind = kind;
    cuuint64_t dims[2] = { static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows) };
    cuuint64_t strides[1] = { static_cast<cuuint64_t>(ld * esize) };
    cuuint32_t box[2] = { static_cast<cuuint32_t>(128 / esize), 128u };
    cuuint32_t estrides[2] = { 1u, 1u };
    CUresult r = get_encode()(&op.map, kind == TcKind::TF32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                            : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16,
                              2, const_cast<void *>(base), dims, strides, box, estrides,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
    {
        throw Error(4, "cuTensorMapEncodeTiled failed with code " + std::to_string(static_cast<int>(r)));
    }
}

void tc_gemm(const TcOperand &A, const TcOperand &B, const TcGemmArgs &args, cudaStream_t s)
{
    if (args.M <= 0 || args.N <= 0)
    {
        return;
    }
    if (A.kind != B.kind)
    {
        throw Error(1, "tc_gemm: A and B must have the same element type");
    }
    const int kstage = (A.kind == TcKind::TF32) ? 32 : 64;
    if (args.K <= 0 || args.K % kstage != 0)
    {
        throw Error(1, "tc_gemm: K must be a positive multiple of " + std::to_string(kstage));
    }
    if ((args.a_col0 % kstage) || (args.b_col0 % kstage) || (args.ldc & 3) ||
        (reinterpret_cast<uintptr_t>(args.C) & 15))
    {
        throw Error(1, "tc_gemm: K offsets must be stage aligned, C 16-byte aligned with ldc % 4 == 0");
    }
    if (args.a_col0 + args.K > A.cols || args.b_col0 + args.K > B.cols || args.a_row0 + args.M > A.rows ||
        args.b_row0 + args.N > B.rows)
    {
        throw Error(1, "tc_gemm: tile range exceeds an operand");
    }
    if (args.lower && args.M != args.N)
    {
        throw Error(1, "tc_gemm: lower mode needs M == N");
    }
    if (args.rowsq != nullptr && (args.N > TN || args.lower || args.rowsq_half < args.M || args.beta != 0.0f))
    {
        throw Error(1, "tc_gemm: rowsq needs N <= 128, beta = 0 and rowsq_half >= M");
    }
    if (args.ldc < args.N)
    {
        throw Error(1, "tc_gemm: ldc must be >= N");
    }
    if (!(args.beta == 0.0f || args.beta == 1.0f))
    {
        throw Error(1, "tc_gemm: beta must be 0 or 1");
    }
    // C as a TMA tensor (FP32, 32 x 32 boxes with 128-byte swizzle) for the
    // epilogue's bulk stores / reduce-adds
    CUtensorMap tmC;
    {
        cuuint64_t dims[2] = { static_cast<cuuint64_t>(args.N), static_cast<cuuint64_t>(args.M) };
        cuuint64_t strides[1] = { static_cast<cuuint64_t>(args.ldc * 4) };
        cuuint32_t box[2] = { 32u, 32u };
        cuuint32_t estrides[2] = { 1u, 1u };
        CUresult r = get_encode()(&tmC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, static_cast<void *>(args.C), dims, strides,
                                  box, estrides, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
        {
            throw Error(4, "cuTensorMapEncodeTiled (C) failed with code " + std::to_string(static_cast<int>(r)));
        }
    }
    // Tile choice: a CTA pair (256 x 256) for large updates, 128 x 256 for wide
    // ones, 128 x 128 for N < 512 (a 256-wide tile would waste up to half its
    // columns there) and for row sums of squares.
    int mode = args.tile_mode;
    if (mode == 0)
    {
        mode = (args.rowsq != nullptr || args.N < 512) ? 1 : (args.M >= 1024 ? 3 : 2);
    }
    if (mode != 1 && args.rowsq != nullptr)
    {
        throw Error(1, "tc_gemm: row sums of squares need the 128 x 128 tile");
    }
    const int sms = sm_count();
    const bool timed = gemm_timing_enabled();
    if (mode == 3)
    {
        const int tiles_m = ceil_div(args.M, 256);
        const int tiles_n = ceil_div(args.N, 256);
        const int ntiles = args.lower ? tiles_m * (tiles_m + 1) / 2 : tiles_m * tiles_n;
        int npairs = std::min(ntiles, sms / 2);
        if (args.max_ctas > 0)
        {
            npairs = std::min(npairs, std::max(1, args.max_ctas / 2));
        }
        if (timed)
        {
            gemm_timing_begin(s);
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * npairs);
        cfg.blockDim = dim3(NUM_THREADS);
        cfg.dynamicSmemBytes = PAIR_SMEM_BYTES;
        cfg.stream = s;
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        attr[1] = programmatic_launch_attr();
        cfg.attrs = attr;
        cfg.numAttrs = 2;
        if (A.kind == TcKind::TF32)
        {
            ensure_smem_attr(reinterpret_cast<const void *>(tc_gemm_pair_kernel<0>), PAIR_SMEM_BYTES);
            GPRAT_CUDA_CHECK(cudaLaunchKernelEx(&cfg, tc_gemm_pair_kernel<0>, A.map, B.map, tmC, args, tiles_n, ntiles));
        }
        else
        {
            ensure_smem_attr(reinterpret_cast<const void *>(tc_gemm_pair_kernel<1>), PAIR_SMEM_BYTES);
            GPRAT_CUDA_CHECK(cudaLaunchKernelEx(&cfg, tc_gemm_pair_kernel<1>, A.map, B.map, tmC, args, tiles_n, ntiles));
        }
    }
    else
    {
        const bool wide = mode == 2;
        const int tnv = wide ? 256 : 128;
        const int tiles_m = ceil_div(args.M, TM);
        const int tiles_n = ceil_div(args.N, tnv);
        int ntiles;
        if (!args.lower)
        {
            ntiles = tiles_m * tiles_n;
        }
        else if (!wide)
        {
            ntiles = tiles_m * (tiles_m + 1) / 2;
        }
        else
        {
            const int a = tiles_m >> 1;
            ntiles = (tiles_m & 1) ? (a + 1) * (a + 1) : a * (a + 1);
        }
        int grid = std::min(ntiles, sms);
        if (args.max_ctas > 0)
        {
            grid = std::min(grid, args.max_ctas);
        }
        if (timed)
        {
            gemm_timing_begin(s);
        }
        auto run = [&](auto kernel, int smem)
        {
            ensure_smem_attr(reinterpret_cast<const void *>(kernel), smem);
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(grid);
            cfg.blockDim = dim3(NUM_THREADS);
            cfg.dynamicSmemBytes = static_cast<size_t>(smem);
            cfg.stream = s;
            cudaLaunchAttribute attr[1] = { programmatic_launch_attr() };
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            GPRAT_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kernel, A.map, B.map, tmC, args, tiles_n, ntiles));
        };
        if (A.kind == TcKind::TF32)
        {
            if (wide)
            {
                run(tc_gemm_kernel<0, 256>, TileCfg<256>::SMEM_BYTES);
            }
            else
            {
                run(tc_gemm_kernel<0, 128>, TileCfg<128>::SMEM_BYTES);
            }
        }
        else
        {
            if (wide)
            {
                run(tc_gemm_kernel<1, 256>, TileCfg<256>::SMEM_BYTES);
            }
            else
            {
                run(tc_gemm_kernel<1, 128>, TileCfg<128>::SMEM_BYTES);
            }
        }
    }
    GPRAT_LAUNCH_CHECK();
    if (timed)
    {
        const double mn = args.lower ? 0.5 * static_cast<double>(args.M) * (args.M + 1)
                                     : static_cast<double>(args.M) * args.N;
        gemm_timing_end(s, 2.0 * mn * args.K);
    }
}

void convert_f64_to_f32(const double *src, int64_t lds, float *dst, int64_t ldd, int rows, int cols, cudaStream_t s)
{
    launch_convert<double>(src, lds, dst, ldd, rows, cols, 0, s);
}

void convert_f32_to_f64(const float *src, int64_t lds, double *dst, int64_t ldd, int rows, int cols, cudaStream_t s)
{
    launch_convert<float>(src, lds, dst, ldd, rows, cols, 1, s);
}

void convert_f32_to_bf16(const float *src, int64_t lds, void *dst, int64_t ldd, int rows, int cols, cudaStream_t s)
{
    launch_convert<float>(src, lds, dst, ldd, rows, cols, 2, s);
}

}  // namespace gprat_cu
