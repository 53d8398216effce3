// Single-launch blocked triangular solves L x = b and L^T x = b (FP64 right-
// hand side; L row-major lower triangle with the inverses of its 128 x 128
// diagonal blocks): the FP64 solves of alpha (trsv_fwd/bwd_fused_kernel) and
// the FP32 solves of the mixed path's preconditioner (trsv_fwd/bwd_f32_kernel,
// further down, which keep their chain in registers).
//
// forward_solve_tiled / backward_solve_tiled (core/src/cpu/tiled_algorithms.cpp:61-115)
// walk the block columns one after another.  Launching one kernel per block
// makes the solve launch-latency bound (two launches per 128 rows).  Here one
// kernel does the whole solve:
//   * the right-hand side is copied aside and x is filled with a sentinel bit
//     pattern (all ones, a NaN no arithmetic produces); every element of x is
//     then written exactly once, by the CTA that solves its block;
//   * every CTA takes a row block by atomic ticket (tickets follow launch
//     order, so a CTA only waits for CTAs that are already running);
//   * before it waits for anything it starts the asynchronous copy of its
//     diagonal inverse into shared memory (lower triangle, packed) and issues
//     the loads of the first tile of L;
//   * it accumulates L_ij x_j over the blocks j it depends on, reading x_j
//     straight from L2 and re-reading an element until it is no longer the
//     sentinel -- the value is the flag, so no fence, counter or extra round
//     trip sits on the chain between two blocks;
//   * x_i = Linv_ii (b_i - sum_j L_ij x_j) from shared memory, eight threads
//     per row.
// L is read exactly once per solve.  Waits are bounded; a wait that runs out
// sets the status word's timeout flag (the caller reports an error).
#include "common.cuh"

namespace gprat_cu
{
namespace
{

constexpr int FT = 256;  // threads per CTA (8 warps)
constexpr int FB = 128;  // block size
constexpr long long SPIN_LIMIT = 1ll << 24;  // with 32 ns sleeps: about 0.5-1 s
// The poll budget the solves use on this device (SPIN_LIMIT unless a test
// shrank it with gprat_cu_test_set_wait_budget).
__device__ long long g_spin_limit = SPIN_LIMIT;
constexpr long long SENTINEL = -1ll;          // 0xFFFF...FF

// Packed lower triangle of a 128 x 128 FP64 block: row r holds columns
// 0..r padded to an even count, so every row starts on a 16-byte boundary.
__host__ __device__ constexpr int packed_off(int r)
{
    return (r >> 1) * (r >> 1) * 2 + 2 * (r >> 1) + (r & 1) * (2 * (r >> 1) + 2);
}
constexpr int PACKED = packed_off(FB);  // 8320 doubles
constexpr size_t SMEM_BYTES = (PACKED + 2 * FB + (FT / 32) * FB) * sizeof(double) + 16;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Starts the copy of Linv_ii's lower triangle into the packed layout.
__device__ __forceinline__ void load_diag_inverse(double *dst, const double *Li)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r = warp; r < FB; r += FT / 32)
    {
        const int pairs = (r + 2) >> 1;
        for (int c2 = lane; c2 < pairs; c2 += 32)
        {
            cp_async16(dst + packed_off(r) + 2 * c2, Li + r * FB + 2 * c2);
        }
    }
}

__device__ __forceinline__ double load_relaxed(const double *p)
{
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}

// Reads N elements of x (one per call site), waiting (bounded) until their
// solvers have written them.  Every lane of the warp calls this together.
// urgent: the block is the one this CTA's own block waits on (its result is
// on the critical path), so every lane re-polls at once; otherwise (the whole
// frontier of waiting CTAs would be polling the same kilobyte of L2) one lane
// polls with a longer sleep and the warp re-reads when it sees data.
template <int N>
__device__ __forceinline__ void await_x(const double *const (&p)[N], double (&v)[N], bool urgent, DeviceStatus *st)
{
    long long spins = 0;
    const long long limit = g_spin_limit;
    for (;;)
    {
        bool missing = false;
#pragma unroll
        for (int q = 0; q < N; ++q)
        {
            v[q] = load_relaxed(p[q]);
            missing |= __double_as_longlong(v[q]) == SENTINEL;
        }
        if (!__any_sync(0xffffffffu, missing))
        {
            return;
        }
        if (++spins > limit)
        {
            if (st != nullptr)
            {
                atomicExch(&st->timeout, 1);
            }
#pragma unroll
            for (int q = 0; q < N; ++q)
            {
                v[q] = 0.0;
            }
            return;
        }
        if (urgent)
        {
            __nanosleep(20);
        }
        else
        {
            // one lane waits on one missing element before the warp re-reads
            const unsigned who = __ballot_sync(0xffffffffu, missing);
            if ((threadIdx.x & 31) == __ffs(who) - 1)
            {
                bool waited = false;
#pragma unroll
                for (int t = 0; t < N; ++t)
                {
                    if (!waited && __double_as_longlong(v[t]) == SENTINEL)
                    {
                        long long inner = 0;
                        while (__double_as_longlong(load_relaxed(p[t])) == SENTINEL && ++inner < limit)
                        {
                            __nanosleep(256);
                        }
                        waited = true;
                    }
                }
            }
            __syncwarp();
        }
    }
}

template <typename T>
__device__ __forceinline__ double to_d(T v)
{
    return static_cast<double>(v);
}

// flags[0] = ticket counter; b = right-hand side (copy); x = solution (sentinel-filled).
template <typename T, typename TI>
__global__ void __launch_bounds__(FT, 1) trsv_fwd_fused_kernel(const T *__restrict__ L, int64_t ld,
                                                               const TI *__restrict__ Linv, int n,
                                                               const double *__restrict__ b, double *x, int *flags,
                                                               DeviceStatus *st)
{
    extern __shared__ __align__(16) double sm[];
    double *linv_s = sm;              // packed lower triangle of Linv_ii
    double *rhs = linv_s + PACKED;    // b_i, then b_i - sum_j L_ij x_j
    int *shared_int = reinterpret_cast<int *>(rhs + 2 * FB + (FT / 32) * FB);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nblk = (n + FB - 1) / FB;
    for (;;)
    {
    if (tid == 0)
    {
        shared_int[0] = atomicAdd(flags, 1);
    }
    __syncthreads();
    const int i = shared_int[0];
    __syncthreads();  // every thread has its ticket before thread 0 draws the next
    if (i >= nblk)
    {
        break;
    }
    const int r0 = i * FB;
    const int bs = min(FB, n - r0);
    load_diag_inverse(linv_s, Linv + static_cast<int64_t>(i) * FB * FB);
    if (tid < FB)
    {
        rhs[tid] = (tid < bs) ? b[r0 + tid] : 0.0;
    }
    __syncthreads();  // rhs rows are updated below by other threads

    // rows warp + 8q of the block; lanes own columns lane + 32c
    constexpr int QB = sizeof(T) == 4 ? 16 : 8;  // rows per batch (registers)
    double part[16];
#pragma unroll
    for (int q = 0; q < 16; ++q)
    {
        part[q] = 0.0;
    }
    for (int j = 0; j < i; ++j)
    {
        const int c0 = j * FB;
#pragma unroll
        for (int qb = 0; qb < 16; qb += QB)
        {
            T v[QB][4];
#pragma unroll
            for (int q = 0; q < QB; ++q)
            {
                const int r = warp + 8 * (qb + q);
                const T *lr = L + static_cast<int64_t>(r0 + min(r, bs - 1)) * ld + c0 + lane;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    v[q][c] = lr[32 * c];
                }
            }
            double xv[4];
            {
                const double *xp[4] = { x + c0 + lane, x + c0 + lane + 32, x + c0 + lane + 64, x + c0 + lane + 96 };
                await_x<4>(xp, xv, j == i - 1, st);
            }
#pragma unroll
            for (int q = 0; q < QB; ++q)
            {
                double s = 0.0;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    s += to_d(v[q][c]) * xv[c];
                }
                part[qb + q] += s;
            }
        }
    }
    // reduce the lane partials of each row
#pragma unroll
    for (int q = 0; q < 16; ++q)
    {
        double s = part[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            s += __shfl_xor_sync(0xffffffffu, s, o);
        }
        part[q] = s;
    }
    if (lane == 0)
    {
#pragma unroll
        for (int q = 0; q < 16; ++q)
        {
            rhs[warp + 8 * q] -= part[q];
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // x_i[r] = sum_{c <= r} Linv[r][c] rhs[c]: eight threads per row, columns
    // p, p+8, ... (consecutive threads read consecutive words), 32 rows per pass
#pragma unroll
    for (int pass = 0; pass < FB / 32; ++pass)
    {
        const int r = pass * 32 + (tid >> 3), p = tid & 7;
        const double *lr = linv_s + packed_off(r);
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < FB / 8; ++k)
        {
            const int c = p + 8 * k;
            s += (c <= r) ? lr[c] * rhs[c] : 0.0;
        }
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        s += __shfl_xor_sync(0xffffffffu, s, 4);
        if (p == 0 && r < bs)
        {
            x[r0 + r] = s;
        }
    }
    __syncthreads();  // shared memory is refilled for the next block
    }
}

template <typename T, typename TI>
__global__ void __launch_bounds__(FT, 1) trsv_bwd_fused_kernel(const T *__restrict__ L, int64_t ld,
                                                               const TI *__restrict__ Linv, int n, int nblk,
                                                               const double *__restrict__ b, double *x, int *flags,
                                                               DeviceStatus *st)
{
    extern __shared__ __align__(16) double sm[];
    double *linv_s = sm;
    double *rhs = linv_s + PACKED;
    double *colpart = rhs + 2 * FB;  // [8][FB]
    int *shared_int = reinterpret_cast<int *>(colpart + (FT / 32) * FB);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (;;)
    {
    if (tid == 0)
    {
        shared_int[0] = nblk - 1 - atomicAdd(flags, 1);
    }
    __syncthreads();
    const int i = shared_int[0];
    __syncthreads();  // every thread has its ticket before thread 0 draws the next
    if (i < 0)
    {
        break;
    }
    const int c0 = i * FB;
    const int bs = min(FB, n - c0);
    load_diag_inverse(linv_s, Linv + static_cast<int64_t>(i) * FB * FB);
    if (tid < FB)
    {
        rhs[tid] = (tid < bs) ? b[c0 + tid] : 0.0;
    }
    // lanes own columns lane + 32c of block i; warps own rows warp + 8q of each block j
    constexpr int QB = sizeof(T) == 4 ? 16 : 8;
    double part[4] = { 0.0, 0.0, 0.0, 0.0 };
    for (int j = nblk - 1; j > i; --j)
    {
        const int r0 = j * FB;
        const int rs = min(FB, n - r0);
#pragma unroll
        for (int qb = 0; qb < 16; qb += QB)
        {
            T v[QB][4];
#pragma unroll
            for (int q = 0; q < QB; ++q)
            {
                const int r = warp + 8 * (qb + q);
                const T *lr = L + static_cast<int64_t>(r0 + min(r, rs - 1)) * ld + c0 + lane;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    v[q][c] = (lane + 32 * c < bs) ? lr[32 * c] : T(0);
                }
            }
            double xv[QB];
            {
                const double *xp[QB];
#pragma unroll
                for (int q = 0; q < QB; ++q)
                {
                    xp[q] = x + r0 + min(warp + 8 * (qb + q), rs - 1);
                }
                await_x<QB>(xp, xv, j == i + 1, st);
            }
#pragma unroll
            for (int q = 0; q < QB; ++q)
            {
                const int r = warp + 8 * (qb + q);
                const double xr = (r < rs) ? xv[q] : 0.0;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    part[c] += to_d(v[q][c]) * xr;
                }
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
    {
        colpart[warp * FB + lane + 32 * c] = part[c];
    }
    __syncthreads();
    if (tid < FB)
    {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < FT / 32; ++w)
        {
            s += colpart[w * FB + tid];
        }
        rhs[tid] -= s;
    }
    cp_async_wait_all();
    __syncthreads();
    // x_i[c] = sum_{p >= c} Linv[p][c] rhs[p]: eight threads per column, rows
    // q, q+8, ..., 32 columns per pass
#pragma unroll
    for (int pass = 0; pass < FB / 32; ++pass)
    {
        const int c = pass * 32 + (tid >> 3), q = tid & 7;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < FB / 8; ++k)
        {
            const int p = q + 8 * k;
            s += (p >= c && p < bs) ? linv_s[packed_off(p) + min(c, p)] * rhs[p] : 0.0;
        }
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        s += __shfl_xor_sync(0xffffffffu, s, 4);
        if (q == 0 && c < bs)
        {
            x[c0 + c] = s;
        }
    }
    __syncthreads();  // shared memory is refilled for the next block
    }
}

// FP32 factor and FP32 inverses (the preconditioner of the mixed path).  The
// chain from one row block to the next runs from registers:
//   * when a CTA takes block i, each thread loads its half row (forward) or
//     half column (backward) of the diagonal inverse into registers and
//     starts cp.async copies of the two nearest off-diagonal tiles (blocks
//     i-2 and i-1 forward, i+2 and i+1 backward) into shared memory, laid
//     out so that the later reads are free of bank conflicts;
//   * the farther blocks are multiplied in FP32 (four products per row and
//     lane) and summed in FP64; the lane partials are reduced into the
//     right-hand side (a reduce-scatter butterfly, 16 shuffles for 16 rows);
//   * each thread moves its part of both near tiles into registers, and one
//     warp stages the two nearest blocks of x in shared memory as they
//     arrive; nothing else waits for the block two steps back, so its
//     arrival costs the chain nothing;
//   * after the neighbour's arrival, 128 FP32 FMAs and one shuffle give each
//     row's (column's) update, and 64 more with the inverse give x_i.
// Products round to FP32 (the preconditioner's accuracy is that of the FP32
// factor); sums over the far blocks stay in FP64.
constexpr int TSTR = 144;  // row stride (floats) of the backward tiles: conflict-free column reads
constexpr size_t SMEM_F32_FWD = 2 * 16 * FT * sizeof(float4) + FB * sizeof(double) + 3 * FB * sizeof(float) + 16;
constexpr size_t SMEM_F32_BWD =
    2 * FB * TSTR * sizeof(float) + (FB + (FT / 32) * FB) * sizeof(double) + 3 * FB * sizeof(float) + 16;

// 64-term FP32 dot product of registers with shared memory (16-byte reads).
__device__ __forceinline__ float dot64(const float (&a)[64], const float *v)
{
    const float4 *v4 = reinterpret_cast<const float4 *>(v);
    float acc[4] = { 0.f, 0.f, 0.f, 0.f };
#pragma unroll
    for (int k4 = 0; k4 < 16; ++k4)
    {
        const float4 q = v4[k4];
        acc[k4 & 3] = fmaf(a[4 * k4], q.x, acc[k4 & 3]);
        acc[k4 & 3] = fmaf(a[4 * k4 + 1], q.y, acc[k4 & 3]);
        acc[k4 & 3] = fmaf(a[4 * k4 + 2], q.z, acc[k4 & 3]);
        acc[k4 & 3] = fmaf(a[4 * k4 + 3], q.w, acc[k4 & 3]);
    }
    return (acc[0] + acc[1]) + (acc[2] + acc[3]);
}

// Sum over the warp of 16 per-lane values: lane l returns the total of value
// (l >> 1) & 15 (a reduce-scatter over lane bits 4..1, then one exchange).
__device__ __forceinline__ double reduce_scatter16(double (&v)[16])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int half = 8, bit = 16; half >= 1; half >>= 1, bit >>= 1)
    {
        const bool hi = (lane & bit) != 0;
#pragma unroll
        for (int t = 0; t < half; ++t)
        {
            const double send = hi ? v[t] : v[t + half];
            const double keep = hi ? v[t + half] : v[t];
            v[t] = keep + __shfl_xor_sync(0xffffffffu, send, bit);
        }
    }
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

__global__ void __launch_bounds__(FT, 1) trsv_fwd_f32_kernel(const float *__restrict__ L, int64_t ld,
                                                             const float *__restrict__ Linv, int n,
                                                             const double *__restrict__ b, double *x, int *flags,
                                                             DeviceStatus *st, const int *skip)
{
    if (skip != nullptr && *skip != 0)
    {
        return;  // every CTA reads the same word: none waits on another
    }
    extern __shared__ __align__(16) double sm[];
    // L_{i,i-2} (tile 0) and L_{i,i-1} (tile 1) in thread-major order:
    // tile[k4][t] = the four floats 64h + 4k4 .. of row t >> 1 (h = t & 1), so
    // thread t reads its half row conflict-free
    float4 *tiles = reinterpret_cast<float4 *>(sm);
    double *rhs = reinterpret_cast<double *>(tiles + 2 * 16 * FT);  // b_i - sum_{j < i-2} L_ij x_j
    float *xs = reinterpret_cast<float *>(rhs + FB);                 // x_{i-2}, x_{i-1}
    float *rs = xs + 2 * FB;                                         // b_i - sum_{j < i} L_ij x_j
    int *shared_int = reinterpret_cast<int *>(rs + FB);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int rr = tid >> 1, h = tid & 1;  // the row and column half of this thread in the products
    const int nblk = (n + FB - 1) / FB;
    for (;;)
    {
    if (tid == 0)
    {
        shared_int[0] = atomicAdd(flags, 1);
    }
    __syncthreads();
    const int i = shared_int[0];
    __syncthreads();  // every thread has its ticket before thread 0 draws the next
    if (i >= nblk)
    {
        break;
    }
    const int r0 = i * FB;
    const int bs = min(FB, n - r0);
    // start the copies of the near tiles: copy m moves chunk k4 = m of thread
    // slot t = tid (consecutive threads fill consecutive 16-byte slots)
#pragma unroll
    for (int t = 0; t < 2; ++t)
    {
        const int j = i - 2 + t;
        if (j >= 0)
        {
            const float *src = L + static_cast<int64_t>(r0 + min(rr, bs - 1)) * ld + j * FB + 64 * h;
#pragma unroll 4
            for (int m = 0; m < 16; ++m)
            {
                cp_async16(tiles + (t * 16 + m) * FT + tid, src + 4 * m);
            }
        }
    }
    // this thread's half row of Linv_ii (zero above the diagonal; defined on
    // rows and columns < bs only)
    float ireg[64];
    {
        const float4 *ip = reinterpret_cast<const float4 *>(Linv + static_cast<int64_t>(i) * FB * FB + rr * FB + 64 * h);
#pragma unroll
        for (int k4 = 0; k4 < 16; ++k4)
        {
            const float4 q = ip[k4];
            ireg[4 * k4] = q.x;
            ireg[4 * k4 + 1] = q.y;
            ireg[4 * k4 + 2] = q.z;
            ireg[4 * k4 + 3] = q.w;
        }
    }
    if (tid < FB)
    {
        rhs[tid] = (tid < bs) ? b[r0 + tid] : 0.0;
    }
    __syncthreads();  // rhs rows are updated below by other threads

    // blocks j < i - 2: rows warp + 8q, lanes own columns lane + 32c, FP64 sums
    double part[16];
#pragma unroll
    for (int q = 0; q < 16; ++q)
    {
        part[q] = 0.0;
    }
    for (int j = 0; j < i - 2; ++j)
    {
        const int c0 = j * FB;
        float v[16][4];
#pragma unroll
        for (int q = 0; q < 16; ++q)
        {
            const int r = warp + 8 * q;
            const float *lr = L + static_cast<int64_t>(r0 + min(r, bs - 1)) * ld + c0 + lane;
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                v[q][c] = lr[32 * c];
            }
        }
        double xv[4];
        {
            const double *xp[4] = { x + c0 + lane, x + c0 + lane + 32, x + c0 + lane + 64, x + c0 + lane + 96 };
            await_x<4>(xp, xv, j == i - 3, st);
        }
        float xf[4];
#pragma unroll
        for (int c = 0; c < 4; ++c)
        {
            xf[c] = static_cast<float>(xv[c]);
        }
#pragma unroll
        for (int q = 0; q < 16; ++q)
        {
            float s2 = v[q][0] * xf[0];
#pragma unroll
            for (int c = 1; c < 4; ++c)
            {
                s2 = fmaf(v[q][c], xf[c], s2);
            }
            part[q] += static_cast<double>(s2);
        }
    }
    if (i > 2)
    {
        const double s2 = reduce_scatter16(part);
        if ((lane & 1) == 0)
        {
            rhs[warp + 8 * ((lane >> 1) & 15)] -= s2;
        }
    }
    cp_async_wait_all();
    __syncthreads();  // tiles landed, rhs complete
    if (bs < FB)
    {
        // a ragged last block: the inverse is defined on rows and columns < bs only
#pragma unroll
        for (int k = 0; k < 64; ++k)
        {
            ireg[k] = (rr < bs && 64 * h + k < bs) ? ireg[k] : 0.f;
        }
    }
    if (i > 0)
    {
        float la[64], lb[64];  // L_{i,i-2} (zero for i = 1) and L_{i,i-1}
#pragma unroll
        for (int k4 = 0; k4 < 16; ++k4)
        {
            const float4 q = tiles[(16 + k4) * FT + tid];
            lb[4 * k4] = q.x;
            lb[4 * k4 + 1] = q.y;
            lb[4 * k4 + 2] = q.z;
            lb[4 * k4 + 3] = q.w;
        }
        if (i > 1)
        {
#pragma unroll
            for (int k4 = 0; k4 < 16; ++k4)
            {
                const float4 q = tiles[k4 * FT + tid];
                la[4 * k4] = q.x;
                la[4 * k4 + 1] = q.y;
                la[4 * k4 + 2] = q.z;
                la[4 * k4 + 3] = q.w;
            }
        }
        else
        {
#pragma unroll
            for (int k = 0; k < 64; ++k)
            {
                la[k] = 0.f;
            }
        }
        if (warp == 0)
        {
#pragma unroll
            for (int t = 0; t < 2; ++t)
            {
                const int j = i - 2 + t;
                double xv[4] = { 0.0, 0.0, 0.0, 0.0 };
                if (j >= 0)
                {
                    const int c0 = j * FB;
                    const double *xp[4] = { x + c0 + lane, x + c0 + lane + 32, x + c0 + lane + 64,
                                            x + c0 + lane + 96 };
                    await_x<4>(xp, xv, true, st);
                }
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    xs[t * FB + lane + 32 * c] = static_cast<float>(xv[c]);
                }
            }
        }
        __syncthreads();  // x_{i-2}, x_{i-1} staged
        float s1 = dot64(la, xs + 64 * h) + dot64(lb, xs + FB + 64 * h);
        s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
        if (h == 0)
        {
            rs[rr] = static_cast<float>(rhs[rr] - static_cast<double>(s1));
        }
    }
    else if (h == 0)
    {
        rs[rr] = static_cast<float>(rhs[rr]);
    }
    __syncthreads();
    float s1 = dot64(ireg, rs + 64 * h);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    if (h == 0 && rr < bs)
    {
        x[r0 + rr] = static_cast<double>(s1);
    }
    __syncthreads();  // shared memory is refilled for the next block
    }
}

__global__ void __launch_bounds__(FT, 1) trsv_bwd_f32_kernel(const float *__restrict__ L, int64_t ld,
                                                             const float *__restrict__ Linv, int n, int nblk,
                                                             const double *__restrict__ b, double *x, int *flags,
                                                             DeviceStatus *st, const int *skip)
{
    if (skip != nullptr && *skip != 0)
    {
        return;
    }
    extern __shared__ __align__(16) double sm[];
    // L_{i+2,i} (tile 0) and L_{i+1,i} (tile 1), row-major with stride TSTR;
    // thread (cc, h) reads column cc, rows 2k + h
    float *tiles = reinterpret_cast<float *>(sm);
    double *rhs = reinterpret_cast<double *>(tiles + 2 * FB * TSTR);  // b_i - sum_{j > i+2} L_ji^T x_j
    double *colpart = rhs + FB;                                         // [8][FB]
    // x_{i+2}, x_{i+1} and the final right-hand side, split by row parity:
    // v[p] at 64 (p & 1) + (p >> 1)
    float *xs = reinterpret_cast<float *>(colpart + (FT / 32) * FB);
    float *rs = xs + 2 * FB;
    int *shared_int = reinterpret_cast<int *>(rs + FB);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cc = tid >> 1, h = tid & 1;  // the column and row parity of this thread in the products
    for (;;)
    {
    if (tid == 0)
    {
        shared_int[0] = nblk - 1 - atomicAdd(flags, 1);
    }
    __syncthreads();
    const int i = shared_int[0];
    __syncthreads();  // every thread has its ticket before thread 0 draws the next
    if (i < 0)
    {
        break;
    }
    const int c0 = i * FB;
    const int bs = min(FB, n - c0);
    // start the copies of the near tiles (16-byte chunks, row by row); block
    // i is full whenever a later block exists
#pragma unroll
    for (int t = 0; t < 2; ++t)
    {
        const int j = i + 2 - t;
        if (j < nblk)
        {
            const int rsj = min(FB, n - j * FB);
#pragma unroll 4
            for (int m = 0; m < 16; ++m)
            {
                const int g = tid + FT * m, row = g >> 5, ch = g & 31;
                cp_async16(tiles + (t * FB + row) * TSTR + 4 * ch,
                           L + static_cast<int64_t>(j * FB + min(row, rsj - 1)) * ld + c0 + 4 * ch);
            }
        }
    }
    // this thread's rows 2k + h of column cc of Linv_ii (zero above the
    // diagonal; defined on rows and columns < bs only)
    float ireg[64];
    {
        const float *ip = Linv + static_cast<int64_t>(i) * FB * FB + cc;
#pragma unroll
        for (int k = 0; k < 64; ++k)
        {
            ireg[k] = ip[(2 * k + h) * FB];
        }
    }
    if (tid < FB)
    {
        rhs[tid] = (tid < bs) ? b[c0 + tid] : 0.0;
    }
    // blocks j > i + 2: lanes own columns lane + 32c of block i, warps rows warp + 8q of block j
    double part[4] = { 0.0, 0.0, 0.0, 0.0 };
    for (int j = nblk - 1; j > i + 2; --j)
    {
        const int r0 = j * FB;
        const int rsj = min(FB, n - r0);
        float v[16][4];
#pragma unroll
        for (int q = 0; q < 16; ++q)
        {
            const int r = warp + 8 * q;
            const float *lr = L + static_cast<int64_t>(r0 + min(r, rsj - 1)) * ld + c0 + lane;
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                v[q][c] = (lane + 32 * c < bs) ? lr[32 * c] : 0.f;
            }
        }
        double xv[16];
        {
            const double *xp[16];
#pragma unroll
            for (int q = 0; q < 16; ++q)
            {
                xp[q] = x + r0 + min(warp + 8 * q, rsj - 1);
            }
            await_x<16>(xp, xv, j == i + 3, st);
        }
        float s2[4] = { 0.f, 0.f, 0.f, 0.f };
#pragma unroll
        for (int q = 0; q < 16; ++q)
        {
            const int r = warp + 8 * q;
            const float xr = (r < rsj) ? static_cast<float>(xv[q]) : 0.f;
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                s2[c] = fmaf(v[q][c], xr, s2[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < 4; ++c)
        {
            part[c] += static_cast<double>(s2[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
    {
        colpart[warp * FB + lane + 32 * c] = part[c];
    }
    cp_async_wait_all();
    __syncthreads();  // tiles landed, column partials written
    if (tid < FB)
    {
        double s2 = 0.0;
#pragma unroll
        for (int w = 0; w < FT / 32; ++w)
        {
            s2 += colpart[w * FB + tid];
        }
        rhs[tid] -= s2;
    }
    if (bs < FB)
    {
        // a ragged last block: the inverse is defined on rows and columns < bs only
#pragma unroll
        for (int k = 0; k < 64; ++k)
        {
            ireg[k] = (cc < bs && 2 * k + h < bs) ? ireg[k] : 0.f;
        }
    }
    if (i + 1 < nblk)
    {
        float la[64], lb[64];  // L_{i+2,i} (zero when block i+2 does not exist) and L_{i+1,i}
#pragma unroll
        for (int k = 0; k < 64; ++k)
        {
            lb[k] = tiles[(FB + 2 * k + h) * TSTR + cc];
        }
        if (i + 2 < nblk)
        {
#pragma unroll
            for (int k = 0; k < 64; ++k)
            {
                la[k] = tiles[(2 * k + h) * TSTR + cc];
            }
        }
        else
        {
#pragma unroll
            for (int k = 0; k < 64; ++k)
            {
                la[k] = 0.f;
            }
        }
        if (warp == 0)
        {
#pragma unroll
            for (int t = 0; t < 2; ++t)
            {
                const int j = i + 2 - t;
                const int rsj = (j < nblk) ? min(FB, n - j * FB) : 0;
                double xv[4] = { 0.0, 0.0, 0.0, 0.0 };
                if (j < nblk)
                {
                    const int r0 = j * FB;
                    const double *xp[4] = { x + r0 + min(lane, rsj - 1), x + r0 + min(lane + 32, rsj - 1),
                                            x + r0 + min(lane + 64, rsj - 1), x + r0 + min(lane + 96, rsj - 1) };
                    await_x<4>(xp, xv, true, st);
                }
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    const int p = lane + 32 * c;
                    xs[t * FB + 64 * (p & 1) + (p >> 1)] = (p < rsj) ? static_cast<float>(xv[c]) : 0.f;
                }
            }
        }
        __syncthreads();  // x_{i+2}, x_{i+1} staged, rhs complete
        float s1 = dot64(la, xs + 64 * h) + dot64(lb, xs + FB + 64 * h);
        s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
        if (h == 0)
        {
            rs[64 * (cc & 1) + (cc >> 1)] = static_cast<float>(rhs[cc] - static_cast<double>(s1));
        }
    }
    else
    {
        __syncthreads();  // rhs complete
        if (h == 0)
        {
            rs[64 * (cc & 1) + (cc >> 1)] = static_cast<float>(rhs[cc]);
        }
    }
    __syncthreads();
    float s1 = dot64(ireg, rs + 64 * h);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    if (h == 0 && cc < bs)
    {
        x[c0 + cc] = static_cast<double>(s1);
    }
    __syncthreads();  // shared memory is refilled for the next block
    }
}

// x: in = b, out = solution.  scratch: n doubles (receives b).
void prepare(double *x, double *scratch, int n, int *flags, cudaStream_t s)
{
    GPRAT_CUDA_CHECK(cudaMemcpyAsync(scratch, x, static_cast<size_t>(n) * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GPRAT_CUDA_CHECK(cudaMemsetAsync(x, 0xFF, static_cast<size_t>(n) * sizeof(double), s));
    GPRAT_CUDA_CHECK(cudaMemsetAsync(flags, 0, sizeof(int), s));
}

// grid: one CTA per row block, or max_ctas (> 0) CTAs that each take row
// blocks by ticket until none is left (the solve then holds fewer SMs).
int grid_for(int nblk, int max_ctas) { return max_ctas > 0 ? std::min(nblk, max_ctas) : nblk; }

template <typename T, typename TI>
void fwd(const T *L, int64_t ld, const TI *Linv, int n, double *x, int *flags, double *scratch, DeviceStatus *st,
         cudaStream_t s, int max_ctas)
{
    const int nblk = ceil_div(n, FB);
    ensure_smem_attr(reinterpret_cast<const void *>(trsv_fwd_fused_kernel<T, TI>), static_cast<int>(SMEM_BYTES));
    prepare(x, scratch, n, flags, s);
    trsv_fwd_fused_kernel<T, TI>
        <<<grid_for(nblk, max_ctas), FT, SMEM_BYTES, s>>>(L, ld, Linv, n, scratch, x, flags, st);
    GPRAT_LAUNCH_CHECK();
}

template <typename T, typename TI>
void bwd(const T *L, int64_t ld, const TI *Linv, int n, double *x, int *flags, double *scratch, DeviceStatus *st,
         cudaStream_t s, int max_ctas)
{
    const int nblk = ceil_div(n, FB);
    ensure_smem_attr(reinterpret_cast<const void *>(trsv_bwd_fused_kernel<T, TI>), static_cast<int>(SMEM_BYTES));
    prepare(x, scratch, n, flags, s);
    trsv_bwd_fused_kernel<T, TI>
        <<<grid_for(nblk, max_ctas), FT, SMEM_BYTES, s>>>(L, ld, Linv, n, nblk, scratch, x, flags, st);
    GPRAT_LAUNCH_CHECK();
}

}  // namespace

void trsv_fused_forward(const double *L, int64_t ld, const double *Linv, int n, double *x, int *flags,
                        double *scratch, DeviceStatus *st, cudaStream_t s, int max_ctas)
{
    fwd(L, ld, Linv, n, x, flags, scratch, st, s, max_ctas);
}

void trsv_fused_backward(const double *L, int64_t ld, const double *Linv, int n, double *x, int *flags,
                         double *scratch, DeviceStatus *st, cudaStream_t s, int max_ctas)
{
    bwd(L, ld, Linv, n, x, flags, scratch, st, s, max_ctas);
}

void trsv_fused_forward_f32(const float *L, int64_t ld, const float *Linv, int n, double *x, int *flags,
                            double *scratch, DeviceStatus *st, cudaStream_t s, int max_ctas, const int *skip)
{
    if ((ld & 3) != 0 || (reinterpret_cast<uintptr_t>(L) & 15) != 0 || (reinterpret_cast<uintptr_t>(Linv) & 15) != 0)
    {
        throw Error(1, "trsv_fused_forward_f32: L and Linv must be 16-byte aligned, ld a multiple of 4");
    }
    const int nblk = ceil_div(n, FB);
    ensure_smem_attr(reinterpret_cast<const void *>(trsv_fwd_f32_kernel), static_cast<int>(SMEM_F32_FWD));
    prepare(x, scratch, n, flags, s);
    trsv_fwd_f32_kernel<<<grid_for(nblk, max_ctas), FT, SMEM_F32_FWD, s>>>(L, ld, Linv, n, scratch, x, flags, st,
                                                                        skip);
    GPRAT_LAUNCH_CHECK();
}

void trsv_fused_backward_f32(const float *L, int64_t ld, const float *Linv, int n, double *x, int *flags,
                             double *scratch, DeviceStatus *st, cudaStream_t s, int max_ctas, const int *skip)
{
    if ((ld & 3) != 0 || (reinterpret_cast<uintptr_t>(L) & 15) != 0 || (reinterpret_cast<uintptr_t>(Linv) & 15) != 0)
    {
        throw Error(1, "trsv_fused_backward_f32: L and Linv must be 16-byte aligned, ld a multiple of 4");
    }
    const int nblk = ceil_div(n, FB);
    ensure_smem_attr(reinterpret_cast<const void *>(trsv_bwd_f32_kernel), static_cast<int>(SMEM_F32_BWD));
    prepare(x, scratch, n, flags, s);
    trsv_bwd_f32_kernel<<<grid_for(nblk, max_ctas), FT, SMEM_F32_BWD, s>>>(L, ld, Linv, n, nblk, scratch, x, flags,
                                                                        st, skip);
    GPRAT_LAUNCH_CHECK();
}

// Sets the poll budget of the solves' waits on the current device; polls < 0
// restores the default.  Test use: a budget of 0 makes a wait on an unsolved
// block give up at once (the status word's timeout flag), with no hang.
void set_trsv_wait_budget(long long polls)
{
    const long long v = polls < 0 ? SPIN_LIMIT : polls;
    GPRAT_CUDA_CHECK(cudaMemcpyToSymbol(g_spin_limit, &v, sizeof(v)));
}

}  // namespace gprat_cu
