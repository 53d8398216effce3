// FP64 matrix products on the int8 tensor cores (Ozaki scheme); the method
// and the slice representation are described in ozaki.cuh.
//
// oz_split_kernel: one CTA per 128 x 128 block of the FP64 source, 8 warps of
// 16 rows; a lane holds 4 consecutive values of a row.  A warp loads its 16
// rows at once into registers (so the block's DRAM latency is paid once, not
// per row), finds the row maxima and, across the CTA, the block maximum,
// and writes s digit planes from the registers, 4 bytes per lane and plane
// (128-byte rows).  Digits
// are peeled with the 1.5 * 2^52 rounding trick: y = t + 1.5 * 2^52 rounds t
// to the nearest integer d (ties to even), d is the low word of y, then
// t <- (t - d) * 254 (t - d is exact; the product rounds only once the
// remainder has used up the 53 bits), so D_0 .. D_{s-1} are the leading s
// balanced base-254 digits of x * 2^(6 - e): |D_0| <= 64, |D_p| <= 127.
//
// oz_gemm_kernel: persistent, warp-specialised CTA pair (cluster of 2, 384
// threads each), one 256 x 128 output tile per pair at a time:
//   warp 0, one lane (both CTAs): TMA producer.  For each 128-column block k
//     and group g it loads digit plane g of A (this CTA's 128 rows, 16 KB)
//     and of B (this CTA's 64 rows, 8 KB) into one slot of a ring of
//     OZ_RING, both counted by the slot's one barrier.  A block's planes stay
//     resident until its last group, so every digit tile crosses from L2
//     once per block; the spare slots let the next block's first planes load
//     while the current block's last groups run.
//   warps 1 and 2, one lane each (leader): MMA issuers, taking alternate
//     groups so that one thread's barrier waits do not idle the tensor core
//     (the issuer below says why).  Group g of block k is one unit:
//     for p = 0..g, four tcgen05.mma.cta_group::2.kind::i8 (M 256, N 128,
//     K 32) of A_p against B_{g-p} into one int32 accumulator in tensor
//     memory (four accumulators of 128 columns rotate); tcgen05.commit frees
//     the accumulator, and after the block (from both issuers) its slots.
//   warps 4..11 (both CTAs): epilogue.  Two warps per TMEM lane quarter, 64
//     columns each (224 registers after setmaxnreg); units are read with
//     double-buffered tcgen05.ld, 16 columns at a time, in pairs of groups
//     (g, g + 1) and combined exactly in int32 as 254 P_g + P_{g+1} (at
//     most 2,112,012,032), converted exactly to FP64 (2^52 + 2^31 bias
//     trick) and added by one FMA with the pair's scale
//     2^(eA + eB - 12) / 254^(g + 1) into 64 FP64 registers per thread (a
//     last unpaired group as 254 P_g at the same scale).  The next block's
//     exponents are loaded while a block is read.  After the tile's last
//     unit, alpha * acc is written from the registers, 8 columns at a time,
//     each lane its own row with 16-byte stores (beta = 1 adds to C; those C
//     values are loaded first); the shared memory a staging transpose would
//     take holds a ninth digit-plane slot instead.
// Every mbarrier wait is bounded (tcgen05_ptx.cuh); a wait that gives up
// raises the CTA's abort flag, the roles leave their loops, TMA copies in
// flight get 200 us to land, the MMA issuer drains, TMEM is freed and the
// status word's timeout flag is set.  No TMA multicast is used.
#include "ozaki.cuh"
#include "tcgen05_ptx.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <string>

namespace gprat_cu
{
namespace
{

using namespace tcx;

constexpr int OZ_ZERO_EXP = -2000;  // an all-zero domain: digits 0
constexpr int OZ_BAD_EXP = 4000;    // a NaN or infinity in the domain: the product becomes NaN
constexpr double RND = 6755399441055744.0;      // 1.5 * 2^52
constexpr double I2D_BIAS = 4503601774854144.0;  // 2^52 + 2^31

__device__ __forceinline__ double pow2(int e)
{
    e = max(-1022, min(1023, e));
    return __longlong_as_double(static_cast<long long>(e + 1023) << 52);
}

// e with max|x| < 2^e over a domain whose maximum is vmax
__device__ __forceinline__ int exp_of(double vmax, bool bad)
{
    if (bad)
    {
        return OZ_BAD_EXP;
    }
    if (vmax == 0.0)
    {
        return OZ_ZERO_EXP;
    }
    const int e = ilogb(vmax) + 1;
    return e < -960 ? OZ_ZERO_EXP : e;
}

// S digit planes of 4 consecutive values (4 bytes per plane at out + p * plane)
template <int S>
__device__ __forceinline__ void write_digits(const double v[4], int e, int8_t *out, int64_t plane)
{
    double t[4];
    const bool zero = (e == OZ_ZERO_EXP || e == OZ_BAD_EXP);
    const double sc = zero ? 0.0 : pow2(6 - e);
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        t[i] = __dmul_rn(v[i], sc);
    }
#pragma unroll
    for (int p = 0; p < S; ++p)
    {
        uint32_t word = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            const double y = __dadd_rn(t[i], RND);
            const int d = __double2loint(y);
            const double r = __dsub_rn(y, RND);
            t[i] = __dmul_rn(__dsub_rn(t[i], r), OZ_BASE);
            word |= (static_cast<uint32_t>(d) & 0xffu) << (8 * i);
        }
        *reinterpret_cast<uint32_t *>(out + p * plane) = word;
    }
}

constexpr int SPLIT_THREADS = 256;

// src is deliberately not __restrict__: loads through a const restrict
// pointer may be compiled as invariant loads, which the compiler is free to
// move above griddepcontrol.wait, before the producing kernel has finished.
template <int S>
__global__ void __launch_bounds__(SPLIT_THREADS) oz_split_kernel(const double *src, int64_t lds, int rows,
                                                                 int8_t *rdig, int64_t rld, int64_t rplane,
                                                                 int32_t *rexp, int rldE, int8_t *bdig, int64_t bld,
                                                                 int64_t bplane, int32_t *bexp, int bldE, int dst_row0,
                                                                 int dst_kb0)
{
    __shared__ double wmax[SPLIT_THREADS / 32];
    __shared__ int wbad[SPLIT_THREADS / 32];
    pdl_wait();
    const int rb = blockIdx.x, kb = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t col = static_cast<int64_t>(kb) * OZ_KB + lane * 4;
    const int r_first = rb * 128 + warp * 16;
    // the warp's 16 rows are loaded at once and kept in registers: the row
    // maxima, the block maximum and the digits all come from these values
    double v[16][4];
#pragma unroll
    for (int i = 0; i < 16; ++i)
    {
        const int r = r_first + i;
        if (r < rows)
        {
            const double2 *p2 = reinterpret_cast<const double2 *>(src + static_cast<int64_t>(r) * lds + col);
            const double2 a = p2[0], b = p2[1];
            v[i][0] = a.x;
            v[i][1] = a.y;
            v[i][2] = b.x;
            v[i][3] = b.y;
        }
        else
        {
            v[i][0] = v[i][1] = v[i][2] = v[i][3] = 0.0;
        }
    }
    int er[16];
    double bm = 0.0;
    bool bbad = false;
#pragma unroll
    for (int i = 0; i < 16; ++i)
    {
        double m = 0.0;
        bool bad = false;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const double av = fabs(v[i][j]);
            bad = bad || !(av <= 1.0e308);
            m = fmax(m, av);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        }
        bad = __any_sync(0xffffffffu, bad);
        er[i] = exp_of(m, bad);
        const int r = r_first + i;
        if (rdig != nullptr && r < rows && lane == 0)
        {
            rexp[static_cast<int64_t>(dst_row0 + r) * rldE + dst_kb0 + kb] = er[i];
        }
        bm = fmax(bm, m);
        bbad = bbad || bad;
    }
    if (lane == 0)
    {
        wmax[warp] = bm;
        wbad[warp] = bbad ? 1 : 0;
    }
    __syncthreads();
    double blk = 0.0;
    bool blkbad = false;
#pragma unroll
    for (int w = 0; w < SPLIT_THREADS / 32; ++w)
    {
        blk = fmax(blk, wmax[w]);
        blkbad = blkbad || wbad[w] != 0;
    }
    const int eb = exp_of(blk, blkbad);
    if (bdig != nullptr && threadIdx.x == 0)
    {
        bexp[static_cast<int64_t>(dst_row0 / 128 + rb) * bldE + dst_kb0 + kb] = eb;
    }
    const int64_t dcol = static_cast<int64_t>(dst_kb0 + kb) * OZ_KB + lane * 4;
#pragma unroll
    for (int i = 0; i < 16; ++i)
    {
        const int r = r_first + i;
        if (r < rows)
        {
            if (rdig != nullptr)
            {
                write_digits<S>(v[i], er[i], rdig + static_cast<int64_t>(dst_row0 + r) * rld + dcol, rplane);
            }
            if (bdig != nullptr)
            {
                write_digits<S>(v[i], eb, bdig + static_cast<int64_t>(dst_row0 + r) * bld + dcol, bplane);
            }
        }
    }
    pdl_launch_dependents();
}

// ---------------------------------------------------------------------------
// GEMM

// warpgroup 0: warp 0 TMA, warps 1 and 2 MMA (warp 3 idle); warpgroups 1 and 2
// (warps 4..11): epilogue.  The kernel launches with 168 registers a thread;
// warpgroup 0 gives registers up (setmaxnreg) so that each epilogue thread
// holds 224: 128 * 56 + 256 * 224 = 384 * 168.
constexpr int OZ_THREADS = 384;
constexpr int OZ_REGS_PRODUCER = 56;
constexpr int OZ_REGS_EPILOGUE = 224;
static_assert(128 * OZ_REGS_PRODUCER + 256 * OZ_REGS_EPILOGUE <= OZ_THREADS * 168,
              "the register split exceeds the registers the block launches with");
constexpr int OZ_EPI_WARPS = 8;
constexpr int OZ_A_BYTES = 128 * 128;  // 128 rows x 128 digit bytes
constexpr int OZ_B_BYTES = 64 * 128;   // this CTA's half of the 128 B rows
constexpr int OZ_RING = 9;  // slots of one A and one B digit plane (>= s + 1: the next block's first planes load early)
constexpr int OZ_NACC = 4;             // int32 accumulators of 128 TMEM columns
constexpr int OZ_TMEM_COLS = OZ_NACC * 128;
constexpr int OZ_SMEM_BYTES =
    1024 + OZ_RING * (OZ_A_BYTES + OZ_B_BYTES) + 512;
static_assert(OZ_SMEM_BYTES <= 232448, "shared memory of the int8 GEMM exceeds the per-CTA limit");
static_assert(OZ_RING >= OZ_MAX_SLICES + 1, "the ring must hold one block's planes plus one");
// D = S32, A and B signed 8-bit, K-major, N = 128, M = 256 (CTA pair)
constexpr uint32_t OZ_IDESC =
    (2u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((256u >> 4) << 24);
constexpr int OZ_GROUP_M = 8;  // row tiles per group of the non-lower tile order

struct OzKernelArgs
{
    int M, N, nkb;
    int a_row0, a_col0, b_row0, b_col0;
    const int32_t *ea;
    int ldea;
    const int32_t *eb;
    int ldeb;
    double *C;
    int64_t ldc;
    double alpha;
    int beta;
    int lower;
    double *rowsq;
    int64_t rowsq_half;
    DeviceStatus *status;
    int groups;
    int tiles_m, tiles_n, ntiles;
    double wpow[OZ_MAX_SLICES + 1];  // wpow[j] = 1 / OZ_BASE^j
};

__device__ __forceinline__ void tma_load_3d_pair(void *dst, const CUtensorMap *map, uint32_t leader_bar, int x, int y,
                                                 int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
        "%5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(leader_bar), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void mma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(OZ_IDESC), "r"(accumulate));
}

__device__ __forceinline__ void tmem_ld16_i(uint32_t taddr, int32_t *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int j = 0; j < 16; ++j)
    {
        v[j] = static_cast<int32_t>(r[j]);
    }
}

// Ties registers written by tcgen05.ld to the point after tcgen05.wait::ld:
// an empty volatile asm that reads and writes each one, so that no use is
// scheduled before the wait.
__device__ __forceinline__ void regs_loaded(int32_t (&v)[16])
{
#pragma unroll
    for (int j = 0; j < 16; ++j)
    {
        asm volatile("" : "+r"(v[j]));
    }
}

// exact int32 -> FP64: the bit pattern 0x43300000:(v ^ 2^31) is 2^52 + 2^31 + v
__device__ __forceinline__ double i2d(int32_t v)
{
    return __dsub_rn(__hiloint2double(0x43300000, v ^ static_cast<int32_t>(0x80000000u)), I2D_BIAS);
}

// pair tile t -> (m0, n0): 256-row x 128-column tiles.  Lower mode: row tile i
// holds the 2 i + 2 column tiles that reach its last row (the final one is
// dropped by the host when it lies right of N).
__device__ __forceinline__ void oz_tile(int t, bool lower, int tiles_m, int tiles_n, int &m0, int &n0)
{
    if (!lower)
    {
        const int span = OZ_GROUP_M * tiles_n;
        const int g = t / span;
        const int first = g * OZ_GROUP_M;
        const int gm = min(tiles_m - first, OZ_GROUP_M);
        const int r = t - g * span;
        m0 = (first + r % gm) * 256;
        n0 = (r / gm) * 128;
        return;
    }
    int i = static_cast<int>((sqrt(4.0 * t + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) <= t)
    {
        ++i;
    }
    while (i > 0 && i * (i + 1) > t)
    {
        --i;
    }
    m0 = i * 256;
    n0 = (t - i * (i + 1)) * 128;
}

__global__ void __launch_bounds__(OZ_THREADS, 1)
    oz_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzKernelArgs p)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *aring = smem;
    uint8_t *bring = aring + OZ_RING * OZ_A_BYTES;
    uint64_t *full = reinterpret_cast<uint64_t *>(bring + OZ_RING * OZ_B_BYTES);
    uint64_t *empty = full + OZ_RING;
    uint64_t *tfull = empty + OZ_RING;
    uint64_t *tempty = tfull + OZ_NACC;
    uint64_t *drain = tempty + OZ_NACC;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1;
    const int npairs = gridDim.x >> 1;
    const int G = p.groups;

    if (threadIdx.x == 0)
    {
        for (int i = 0; i < OZ_RING; ++i)
        {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 2);  // one commit from each MMA issuer
        }
        for (int u = 0; u < OZ_NACC; ++u)
        {
            mbar_init(&tfull[u], 1);
            mbar_init(&tempty[u], 2 * OZ_EPI_WARPS);
        }
        mbar_init(drain, 2);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::);
    }
    tc_fence_before();
    cluster_sync_all();  // barriers of both CTAs initialised, TMEM allocated
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    pdl_wait();  // the previous kernel's results are visible from here on
    if (warp < 4)
    {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(OZ_REGS_PRODUCER));
    }
    if (warp == 0)
    {
        if (lane == 0)
        {
            // ---------------- TMA producer (both CTAs) ----------------
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
            int n = 0;  // digit-plane pairs loaded
            bool ok = true;
            for (int t = pair; ok && t < p.ntiles; t += npairs)
            {
                int m0, n0;
                oz_tile(t, p.lower != 0, p.tiles_m, p.tiles_n, m0, n0);
                const int arow = p.a_row0 + m0 + 128 * static_cast<int>(rank);
                const int brow = p.b_row0 + n0 + 64 * static_cast<int>(rank);
                for (int kb = 0; ok && kb < p.nkb; ++kb)
                {
                    const int xa = p.a_col0 + kb * OZ_KB, xb = p.b_col0 + kb * OZ_KB;
                    for (int g = 0; ok && g < G; ++g)
                    {
                        // slot n % OZ_RING takes A_g and B_g; one barrier counts both
                        const int slot = n % OZ_RING;
                        if (!mbar_wait(&empty[slot], ((n / OZ_RING) & 1u) ^ 1u, abort_flag))
                        {
                            ok = false;
                            break;
                        }
                        if (leader)
                        {
                            mbar_expect_tx(&full[slot], 2 * (OZ_A_BYTES + OZ_B_BYTES));  // both CTAs' bytes
                        }
                        const uint32_t bar = map_to_rank(&full[slot], 0);
                        tma_load_3d_pair(aring + slot * OZ_A_BYTES, &tmA, bar, xa, arow, g);
                        tma_load_3d_pair(bring + slot * OZ_B_BYTES, &tmB, bar, xb, brow, g);
                        ++n;
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
    else if (warp == 1 || warp == 2)
    {
        if (lane == 0 && leader)
        {
            // ---------------- MMA issuers (leader only, two threads) ----------------
            // An issuing thread runs in step with the tensor core (an MMA issue
            // returns about when the previous one completes), and a barrier
            // test in that thread costs a shared-memory round trip, which is
            // slow while the tensor core streams its operands; the tensor core
            // would sit idle for it.  Two threads (warps 1 and 2) therefore
            // issue: groups of even global index from one, odd from the other
            // (so each owns two of the four accumulators), and while one waits
            // the other's MMAs keep the tensor core busy.  Before a group a
            // thread waits for its accumulator and for the digit planes of
            // the block it has not seen yet; after the block both threads
            // commit to each slot's empty barrier (count 2).  Descriptors
            // advance from the ring bases (a slot is OZ_A_BYTES / 16 or
            // OZ_B_BYTES / 16 units of the descriptor's address field).
            const int me = warp - 1;
            const uint64_t adesc0 = sw128_desc(smem_u32(aring));
            const uint64_t bdesc0 = sw128_desc(smem_u32(bring));
            int n = 0, nu = 0;
            bool ok = true;
            for (int t = pair; ok && t < p.ntiles; t += npairs)
            {
                for (int kb = 0; ok && kb < p.nkb; ++kb)
                {
                    const int s0 = n % OZ_RING;  // slot of this block's plane 0
                    int seen = -1;               // planes of this block this thread has waited for
                    for (int g = 0; ok && g < G; ++g, ++nu)
                    {
                        if ((nu & 1) != me)
                        {
                            continue;
                        }
                        const int u = nu % OZ_NACC;
                        if (nu >= OZ_NACC && !mbar_wait(&tempty[u], ((nu / OZ_NACC) & 1u) ^ 1u, abort_flag))
                        {
                            ok = false;
                            break;
                        }
                        for (int pl = seen + 1; ok && pl <= g; ++pl)
                        {
                            const int ni = n + pl;
                            ok = mbar_wait(&full[ni % OZ_RING], (ni / OZ_RING) & 1u, abort_flag);
                        }
                        if (!ok)
                        {
                            break;
                        }
                        seen = g;
                        tc_fence_after();
                        const uint32_t d = tmem_base + static_cast<uint32_t>(u * 128);
                        int aslot = s0;      // slot of A_pa
                        int bslot = s0 + g;  // slot of B_{g-pa}
                        bslot -= bslot >= OZ_RING ? OZ_RING : 0;
                        for (int pa = 0; pa <= g; ++pa)  // A plane pa against B plane g - pa
                        {
                            const uint64_t adesc = adesc0 + static_cast<uint64_t>(aslot * (OZ_A_BYTES >> 4));
                            const uint64_t bdesc = bdesc0 + static_cast<uint64_t>(bslot * (OZ_B_BYTES >> 4));
#pragma unroll
                            for (int kk = 0; kk < 4; ++kk)
                            {
                                // 32 bytes of K per instruction: advance the start address by 2 x 16 B
                                mma_i8_pair(d, adesc + 2 * kk, bdesc + 2 * kk, (pa | kk) != 0 ? 1u : 0u);
                            }
                            aslot = aslot + 1 == OZ_RING ? 0 : aslot + 1;
                            bslot = bslot == 0 ? OZ_RING - 1 : bslot - 1;
                        }
                        mma_commit_pair_both(&tfull[u]);
                    }
                    if (!ok)
                    {
                        break;
                    }
                    // a slot is free once both threads' MMAs of this block complete
                    for (int pa = 0; pa < G; ++pa)
                    {
                        const int sl = s0 + pa;
                        mma_commit_pair_both(&empty[sl >= OZ_RING ? sl - OZ_RING : sl]);
                    }
                    n += G;
                }
            }
            // drain (count 2): completes once every MMA both threads issued has completed
            mma_commit_pair_local(drain);
            mbar_wait(drain, 0u, abort_flag);
        }
    }
    else if (warp >= 4)
    {
        // ---------------- epilogue (warps 4..11 of both CTAs) ----------------
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(OZ_REGS_EPILOGUE));
        const int ew = warp - 4;
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        const int h = ew >> 2;   // column half
        int nu = 0;
        bool ok = true;
        for (int t = pair; ok && t < p.ntiles; t += npairs)
        {
            int mp, n0;
            oz_tile(t, p.lower != 0, p.tiles_m, p.tiles_n, mp, n0);
            const int row0w = mp + 128 * static_cast<int>(rank) + q * 32;  // this warp's first row of C
            const int row = row0w + lane;
            const bool rvalid = row < p.M;
            const int32_t *earow = p.ea + static_cast<int64_t>(p.a_row0 + (rvalid ? row : 0)) * p.ldea + p.a_col0 / OZ_KB;
            const int32_t *ebblk = p.eb + static_cast<int64_t>((p.b_row0 + n0) / 128) * p.ldeb + p.b_col0 / OZ_KB;
            double acc[64];
#pragma unroll
            for (int j = 0; j < 64; ++j)
            {
                acc[j] = 0.0;
            }
            int ea_next = earow[0], eb_next = ebblk[0];
            for (int kb = 0; ok && kb < p.nkb; ++kb)
            {
                const int ea = ea_next;
                const int eb = eb_next;
                if (kb + 1 < p.nkb)
                {
                    // the next block's exponents load while this block's groups are read
                    ea_next = earow[kb + 1];
                    eb_next = ebblk[kb + 1];
                }
                const bool bad = ea == OZ_BAD_EXP || eb == OZ_BAD_EXP;
                // groups in pairs (g, g + 1): OZ_BASE P_g + P_{g+1} is exact in int32
                // (at most 2,112,012,032 for the pair (4, 5), the largest), so one
                // conversion and one FMA serve both
                for (int g = 0; g < G; g += 2)
                {
                    const bool two = g + 1 < G;
                    const int u0 = nu % OZ_NACC;
                    const int u1 = (nu + 1) % OZ_NACC;
                    if (!mbar_wait(&tfull[u0], (nu / OZ_NACC) & 1u, abort_flag) ||
                        (two && !mbar_wait(&tfull[u1], ((nu + 1) / OZ_NACC) & 1u, abort_flag)))
                    {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t lane_base = tmem_base + (static_cast<uint32_t>(q * 32) << 16) +
                                               static_cast<uint32_t>(h * 64);
                    const uint32_t t0 = lane_base + static_cast<uint32_t>(u0 * 128);
                    const uint32_t t1 = lane_base + static_cast<uint32_t>(u1 * 128);
                    // a last unpaired group counts as OZ_BASE P_g + 0 at the pair's scale
                    const double sc = bad ? __longlong_as_double(0x7ff8000000000000ll)
                                          : pow2(ea + eb - 12) * p.wpow[g + 1];
                    // 16 columns of each group at a time, double-buffered: the next
                    // chunk's tensor-memory loads are in flight while this chunk converts
                    auto chunk = [&](int32_t(&v)[16], int32_t(&w)[16], int32_t(&vn)[16], int32_t(&wn)[16], int c)
                    {
                        tmem_ld_wait();
                        regs_loaded(v);
                        regs_loaded(w);
                        if (c < 3)
                        {
                            tmem_ld16_i(t0 + (c + 1) * 16, vn);
                            if (two)
                            {
                                tmem_ld16_i(t1 + (c + 1) * 16, wn);
                            }
                            else
                            {
#pragma unroll
                                for (int k = 0; k < 16; ++k)
                                {
                                    wn[k] = 0;
                                }
                            }
                        }
                        else
                        {
                            // both accumulators are read: the MMA warp may reuse them
                            tc_fence_before();
                            __syncwarp();
                            if (lane == 0)
                            {
                                mbar_arrive_remote(map_to_rank(&tempty[u0], 0));
                                if (two)
                                {
                                    mbar_arrive_remote(map_to_rank(&tempty[u1], 0));
                                }
                            }
                        }
#pragma unroll
                        for (int k = 0; k < 16; ++k)
                        {
                            acc[c * 16 + k] = fma(i2d(v[k] * OZ_IBASE + w[k]), sc, acc[c * 16 + k]);
                        }
                    };
                    int32_t va[16], wa[16], vb[16], wb[16];
                    tmem_ld16_i(t0, va);
                    if (two)
                    {
                        tmem_ld16_i(t1, wa);
                    }
                    else
                    {
#pragma unroll
                        for (int k = 0; k < 16; ++k)
                        {
                            wa[k] = 0;
                        }
                    }
                    chunk(va, wa, vb, wb, 0);
                    chunk(vb, wb, va, wa, 1);
                    chunk(va, wa, vb, wb, 2);
                    chunk(vb, wb, va, wa, 3);
                    nu += two ? 2 : 1;
                }
            }
            if (!ok)
            {
                break;
            }
            // ---- write alpha * acc: each lane its own row, 8 columns at a time ----
            // 16-byte stores straight from the registers (no shared-memory
            // staging, which leaves its space to the digit-plane ring); with
            // beta = 1 the 8 columns' C values are loaded first.
            double sq = 0.0;
            double *crow = p.C + static_cast<int64_t>(rvalid ? row : 0) * p.ldc;
#pragma unroll
            for (int c = 0; c < 8; ++c)
            {
                const int col0 = n0 + h * 64 + c * 8;
                // warp-uniform: chunk right of C, below C, or (lower) above the diagonal for all rows
                if (col0 >= p.N || row0w >= p.M || (p.lower && col0 > row0w + 31))
                {
                    continue;
                }
                double2 cold[4];
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    const int gc = col0 + 2 * j;
                    const bool full = rvalid && gc + 1 < p.N && (!p.lower || gc + 1 <= row);
                    cold[j] = (p.beta && full) ? *reinterpret_cast<const double2 *>(crow + gc) : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    const int gc = col0 + 2 * j;
                    const double x = p.alpha * acc[c * 8 + 2 * j];
                    const double y = p.alpha * acc[c * 8 + 2 * j + 1];
                    if (p.rowsq != nullptr && rvalid)
                    {
                        if (gc < p.N)
                        {
                            sq += x * x;
                        }
                        if (gc + 1 < p.N)
                        {
                            sq += y * y;
                        }
                    }
                    if (!rvalid)
                    {
                        continue;
                    }
                    const bool ok0 = gc < p.N && (!p.lower || gc <= row);
                    const bool ok1 = gc + 1 < p.N && (!p.lower || gc + 1 <= row);
                    if (ok0 && ok1)
                    {
                        double2 o = make_double2(x, y);
                        if (p.beta)
                        {
                            o.x += cold[j].x;
                            o.y += cold[j].y;
                        }
                        *reinterpret_cast<double2 *>(crow + gc) = o;
                    }
                    else if (ok0)
                    {
                        crow[gc] = p.beta ? crow[gc] + x : x;
                    }
                }
            }
            __syncwarp();
            if (p.rowsq != nullptr && rvalid)
            {
                p.rowsq[h * p.rowsq_half + row] += sq;  // single writer per word and launch
            }
        }
        // the CTA's last tile is written: the next kernel in the stream may
        // start its set-up
        pdl_launch_dependents();
    }

    tc_fence_before();
    cluster_sync_all();  // no CTA leaves while its peer may still signal or read it
    if (warp == 0)
    {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(OZ_TMEM_COLS));
    }
    if (threadIdx.x == 0 && *abort_flag && p.status != nullptr)
    {
        atomicExch(&p.status->timeout, 1);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once,
                   []
                   {
                       void *q = nullptr;
                       cudaDriverEntryPointQueryResult r;
                       if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &q, 12000, cudaEnableDefault,
                                                            &r) == cudaSuccess &&
                           r == cudaDriverEntryPointSuccess)
                       {
                           fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(q);
                       }
                   });
    if (fn == nullptr)
    {
        throw Error(4, "cuTensorMapEncodeTiled is not available from the driver");
    }
    return fn;
}

void encode_digits(CUtensorMap *map, int8_t *base, int rows, int cols, int64_t ld, int64_t plane, int s, int box_rows)
{
    cuuint64_t dims[3] = { static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows), static_cast<cuuint64_t>(s) };
    cuuint64_t strides[2] = { static_cast<cuuint64_t>(ld), static_cast<cuuint64_t>(plane) };
    cuuint32_t box[3] = { 128u, static_cast<cuuint32_t>(box_rows), 1u };
    cuuint32_t estrides[3] = { 1u, 1u, 1u };
    CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estrides,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
    {
        throw Error(4, "cuTensorMapEncodeTiled (digit planes) failed with code " + std::to_string(static_cast<int>(r)));
    }
}

}  // namespace

void oz_make_operand(OzOperand &op, int8_t *digits, int32_t *exps, int rows, int cols, int64_t ld, int64_t plane,
                     int ldE, int s, bool block)
{
    if (digits == nullptr || exps == nullptr || rows <= 0 || cols <= 0 || cols % OZ_KB != 0 || ld < cols ||
        ld % OZ_KB != 0 || plane < static_cast<int64_t>(rows) * ld || plane % 16 != 0 || ldE < cols / OZ_KB ||
        s < OZ_MIN_SLICES || s > OZ_MAX_SLICES || (reinterpret_cast<uintptr_t>(digits) & 127))
    {
        throw Error(1, "oz_make_operand: invalid digit-plane layout");
    }
    op.digits = digits;
    op.exps = exps;
    op.rows = rows;
    op.cols = cols;
    op.ld = ld;
    op.plane = plane;
    op.ldE = ldE;
    op.s = s;
    op.block = block;
    encode_digits(&op.map_a, digits, rows, cols, ld, plane, s, 128);
    encode_digits(&op.map_b, digits, rows, cols, ld, plane, s, 64);
}

void oz_split(const double *src, int64_t lds, int rows, int cols, const OzOperand *row_op, const OzOperand *blk_op,
              int dst_row0, int dst_col0, cudaStream_t s)
{
    if (rows <= 0 || cols <= 0)
    {
        return;
    }
    if (cols % OZ_KB != 0 || dst_col0 % OZ_KB != 0 || (lds & 1) || (reinterpret_cast<uintptr_t>(src) & 15) ||
        (row_op == nullptr && blk_op == nullptr))
    {
        throw Error(1, "oz_split: cols and dst_col0 must be multiples of 128, src 16-byte aligned with an even ld");
    }
    const int slices = row_op != nullptr ? row_op->s : blk_op->s;
    for (const OzOperand *op : { row_op, blk_op })
    {
        if (op == nullptr)
        {
            continue;
        }
        if (op->s != slices || dst_row0 < 0 || dst_row0 + rows > op->rows || dst_col0 + cols > op->cols)
        {
            throw Error(1, "oz_split: destination range exceeds the slice operand");
        }
    }
    if (blk_op != nullptr && dst_row0 % 128 != 0)
    {
        throw Error(1, "oz_split: block exponents need dst_row0 to be a multiple of 128");
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ceil_div(rows, 128), cols / OZ_KB);
    cfg.blockDim = dim3(SPLIT_THREADS);
    cfg.stream = s;
    cudaLaunchAttribute attr[1] = { programmatic_launch_attr() };
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void (*kern)(const double *, int64_t, int, int8_t *, int64_t, int64_t, int32_t *, int, int8_t *, int64_t,
                 int64_t, int32_t *, int, int, int) = nullptr;
    switch (slices)
    {
    case 3: kern = oz_split_kernel<3>; break;
    case 4: kern = oz_split_kernel<4>; break;
    case 5: kern = oz_split_kernel<5>; break;
    case 6: kern = oz_split_kernel<6>; break;
    case 7: kern = oz_split_kernel<7>; break;
    default: throw Error(1, "oz_split: unsupported digit-plane count");
    }
    static_assert(OZ_MAX_SLICES == 7 && OZ_MIN_SLICES == 3, "oz_split instantiates 3..7 digit planes");
    GPRAT_CUDA_CHECK(cudaLaunchKernelEx(
        &cfg, kern, src, lds, rows, row_op ? row_op->digits : static_cast<int8_t *>(nullptr),
        row_op ? row_op->ld : int64_t(0), row_op ? row_op->plane : int64_t(0),
        row_op ? row_op->exps : static_cast<int32_t *>(nullptr), row_op ? row_op->ldE : 0,
        blk_op ? blk_op->digits : static_cast<int8_t *>(nullptr), blk_op ? blk_op->ld : int64_t(0),
        blk_op ? blk_op->plane : int64_t(0), blk_op ? blk_op->exps : static_cast<int32_t *>(nullptr),
        blk_op ? blk_op->ldE : 0, dst_row0, dst_col0 / OZ_KB));
    GPRAT_LAUNCH_CHECK();
}

void oz_gemm(const OzOperand &A, const OzOperand &B, const OzGemmArgs &a, cudaStream_t s)
{
    if (a.M <= 0 || a.N <= 0)
    {
        return;
    }
    if (A.block || !B.block || A.s != B.s)
    {
        throw Error(1, "oz_gemm: A must be a row operand and B a block operand with the same slice count");
    }
    const int G = a.groups == 0 ? A.s : a.groups;
    if (G < 1 || G > A.s)
    {
        throw Error(1, "oz_gemm: groups must be in [1, s]");
    }
    if (a.K <= 0 || a.K % OZ_KB != 0 || a.a_col0 % OZ_KB != 0 || a.b_col0 % OZ_KB != 0 || a.b_row0 % 128 != 0 ||
        a.a_row0 < 0 || a.b_row0 < 0)
    {
        throw Error(1, "oz_gemm: K, a_col0, b_col0 and b_row0 must be multiples of 128");
    }
    if (a.a_row0 + a.M > A.rows || a.b_row0 + a.N > B.rows || a.a_col0 + a.K > A.cols || a.b_col0 + a.K > B.cols)
    {
        throw Error(1, "oz_gemm: range exceeds an operand");
    }
    if (a.C == nullptr || (reinterpret_cast<uintptr_t>(a.C) & 15) || (a.ldc & 1) || a.ldc < a.N)
    {
        throw Error(1, "oz_gemm: C must be 16-byte aligned with an even ldc >= N");
    }
    if (!(a.beta == 0.0 || a.beta == 1.0))
    {
        throw Error(1, "oz_gemm: beta must be 0 or 1");
    }
    if (a.lower && a.M != a.N)
    {
        throw Error(1, "oz_gemm: lower mode needs M == N");
    }
    if (a.rowsq != nullptr && (a.lower || a.beta != 0.0 || a.rowsq_half < a.M))
    {
        throw Error(1, "oz_gemm: rowsq needs beta = 0, no lower mode and rowsq_half >= M");
    }
    OzKernelArgs k{};
    k.M = a.M;
    k.N = a.N;
    k.nkb = a.K / OZ_KB;
    k.a_row0 = a.a_row0;
    k.a_col0 = a.a_col0;
    k.b_row0 = a.b_row0;
    k.b_col0 = a.b_col0;
    k.ea = A.exps;
    k.ldea = A.ldE;
    k.eb = B.exps;
    k.ldeb = B.ldE;
    k.C = a.C;
    k.ldc = a.ldc;
    k.alpha = a.alpha;
    k.beta = a.beta != 0.0 ? 1 : 0;
    k.lower = a.lower ? 1 : 0;
    k.rowsq = a.rowsq;
    k.rowsq_half = a.rowsq_half;
    k.status = a.status;
    k.groups = G;
    double pw = 1.0;
    for (int j = 0; j <= OZ_MAX_SLICES; ++j)
    {
        k.wpow[j] = 1.0 / pw;  // OZ_BASE^j is exact up to j = 6
        pw *= OZ_BASE;
    }
    k.tiles_m = ceil_div(a.M, 256);
    k.tiles_n = ceil_div(a.N, 128);
    if (a.lower)
    {
        k.ntiles = k.tiles_m * (k.tiles_m + 1) - (2 * k.tiles_m > k.tiles_n ? 1 : 0);
    }
    else
    {
        k.ntiles = k.tiles_m * k.tiles_n;
    }
    const int sms = device_sm_count();
    int npairs = std::min(k.ntiles, sms / 2);
    if (a.max_ctas > 0)
    {
        npairs = std::min(npairs, std::max(1, a.max_ctas / 2));
    }
    const bool timed = gemm_timing_enabled();
    if (timed)
    {
        gemm_timing_begin(s);
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * npairs);
    cfg.blockDim = dim3(OZ_THREADS);
    cfg.dynamicSmemBytes = OZ_SMEM_BYTES;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1] = programmatic_launch_attr();
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    ensure_smem_attr(reinterpret_cast<const void *>(oz_gemm_kernel), OZ_SMEM_BYTES);
    GPRAT_CUDA_CHECK(cudaLaunchKernelEx(&cfg, oz_gemm_kernel, A.map_a, B.map_b, k));
    GPRAT_LAUNCH_CHECK();
    if (timed)
    {
        // int8 tensor-core operations issued (the pipe this kernel is bound by)
        const double mn = a.lower ? 0.5 * static_cast<double>(a.M) * (a.M + 1) : static_cast<double>(a.M) * a.N;
        gemm_timing_end(s, 2.0 * mn * a.K * (G * (G + 1) / 2));
    }
}

}  // namespace gprat_cu
