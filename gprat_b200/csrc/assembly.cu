// Squared-exponential covariance assembly on sm_100a.
//
// k(z_i, z_j) = v * exp(-0.5 / l^2 * sum_k (z_{i+k} - z_{j+k})^2): feature
// rows are sliding windows of one series (compute_covariance_function,
// core/src/cpu/gp_algorithms.cpp:11-28; GPU twin core/src/gpu/gp_algorithms.cu:16-55).
//
// One CTA produces a 64-row x 128-column block.  The two windows of the
// series it needs (64+d-1 and 128+d-1 values) are staged in shared memory
// once; each thread owns one column and walks the rows, so row values are
// shared-memory broadcasts and column values are conflict-free.  Every row of
// the block is written by whole warps as contiguous 256-byte segments
// (coalesced).
//
// Distances.  For d < 16 every entry sums its d squares directly, in the
// reference's order and rounding (separate multiply and add, k ascending), so
// entries differ from the reference only by exp()'s last-place rounding.  For
// d >= 16 the sliding windows give an O(1) update along each diagonal,
//   D(i, j) = D(i-1, j-1) - (x_{i-1} - x_{j-1})^2 + (x_{i+d-1} - x_{j+d-1})^2,
// so only the block's first row and the first column of each warp are summed
// directly (d terms); the other entries take the left neighbour's previous-row
// distance by shuffle.  The drift over at most 63 steps is ~1e-14 of D.
// Per-row windows (row_offsets, a serving batch) always sum directly, so an
// entry does not depend on where its row falls in a batch.
#include "common.cuh"

namespace gprat_cu
{
namespace
{

constexpr int AR = 64;   // rows per CTA
constexpr int AC = 128;  // columns per CTA (= threads)
constexpr int RB = 4;    // rows per inner pass

__device__ __forceinline__ double se_entry(double dist, double neg_half_inv_l2, double v)
{
    return v * exp(__dmul_rn(neg_half_inv_l2, dist));
}

// Computes RB distances for rows i..i+RB-1 (local) and column j (local).
// Row r's window starts at xr[r * rs]: rs = 1 for the sliding window of one
// series, rs = d when every row's window was staged separately.
__device__ __forceinline__ void distances(const double *xr, const double *xc, int i, int j, int d, int rs,
                                          double (&acc)[RB])
{
#pragma unroll
    for (int r = 0; r < RB; ++r)
    {
        acc[r] = 0.0;
    }
    for (int k = 0; k < d; ++k)
    {
        double c = xc[j + k];
#pragma unroll
        for (int r = 0; r < RB; ++r)
        {
            double z = __dsub_rn(xr[(i + r) * rs + k], c);
            acc[r] = __dadd_rn(acc[r], __dmul_rn(z, z));
        }
    }
}

// Direct distance of local row i (window at xr[i * rs]) and local column j.
__device__ __forceinline__ double distance1(const double *xr, const double *xc, int i, int j, int d, int rs)
{
    double acc = 0.0;
    for (int k = 0; k < d; ++k)
    {
        const double z = __dsub_rn(xr[i * rs + k], xc[j + k]);
        acc = __dadd_rn(acc, __dmul_rn(z, z));
    }
    return acc;
}

constexpr int RECUR_MIN_D = 16;

// mode 0: K (lower tiles of size T incl. full diagonal tiles, + noise on the
//         global diagonal); mode 1: cross / prior (all entries, no noise).
// out32 (optional): the same entries rounded to FP32 (mixed path).
template <int MODE, typename OutT>
__global__ void __launch_bounds__(AC) se_kernel(const double *__restrict__ xrow,
                                               int rows,
                                               const double *__restrict__ xcol,
                                               int cols,
                                               int d,
                                               int T,
                                               const DeviceParams *__restrict__ p,
                                               OutT *__restrict__ out,
                                               int64_t ldo,
                                               const double *__restrict__ alpha,
                                               double *__restrict__ mean_partial,
                                               int mean_parts,
                                               const int64_t *__restrict__ row_offsets,
                                               float *__restrict__ out32,
                                               int64_t ld32)
{
    extern __shared__ double sh[];
    const int i0 = blockIdx.y * AR;
    const int j0 = blockIdx.x * AC;
    if (MODE == 0)
    {
        int last_row = min(i0 + AR, rows) - 1;
        int max_col = (last_row / T + 1) * T - 1;
        if (j0 > max_col)
        {
            return;
        }
    }
    // Row windows: the sliding window of one series (xr[r .. r+d-1]), or, with
    // row_offsets, each row's own window xrow[row_offsets[g] ..] staged at xr[r*d].
    const int rs = (row_offsets != nullptr) ? d : 1;
    const int xr_size = (row_offsets != nullptr) ? AR * d : AR + d;
    double *xr = sh;                 // xr_size
    double *xc = sh + xr_size;       // AC + d - 1
    double *red = xc + AC + d;       // AR x (AC/32) mean partials
    double *bnd = red + AR * (AC / 32);  // AR x (AC/32): direct distances of each warp's first column
    if (row_offsets != nullptr)
    {
        for (int q = threadIdx.x; q < AR * d; q += AC)
        {
            const int r = q / d, k = q % d;
            const int g = i0 + r;
            xr[q] = (g < rows) ? xrow[row_offsets[g] + k] : 0.0;
        }
    }
    else
    {
        for (int q = threadIdx.x; q < AR + d - 1; q += AC)
        {
            int g = i0 + q;
            xr[q] = (g < rows + d - 1) ? xrow[g] : 0.0;
        }
    }
    for (int q = threadIdx.x; q < AC + d - 1; q += AC)
    {
        int g = j0 + q;
        xc[q] = (g < cols + d - 1) ? xcol[g] : 0.0;
    }
    // mode 0: first column past the tile of each row (one division per row, not per entry)
    __shared__ int rowlim[AR];
    if (MODE == 0 && threadIdx.x < AR)
    {
        rowlim[threadIdx.x] = ((i0 + threadIdx.x) / T + 1) * T;
    }
    __syncthreads();

    const double l = p->hyper[0];
    const double v = p->hyper[1];
    const double noise = p->hyper[2];
    const double nh = -0.5 / (l * l);
    const int j = threadIdx.x;
    const int gj = j0 + j;
    const double aj = (alpha != nullptr && gj < cols) ? alpha[gj] : 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    const bool recur = d >= RECUR_MIN_D && row_offsets == nullptr;
    auto emit = [&](int r, double dist)
    {
        const int gi = i0 + r;
        double val = se_entry(dist, nh, v);
        bool inside = gi < rows && gj < cols;
        if (MODE == 0)
        {
            inside = inside && (gj < rowlim[r]);  // tile of column gj at or left of gi's tile
            if (gi == gj)
            {
                val += noise;
            }
        }
        if (inside && out != nullptr)
        {
            out[static_cast<int64_t>(gi) * ldo + gj] = static_cast<OutT>(val);
        }
        if (inside && out32 != nullptr)
        {
            out32[static_cast<int64_t>(gi) * ld32 + gj] = static_cast<float>(val);
        }
        if (mean_partial != nullptr)
        {
            double prod = inside ? val * aj : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
            {
                prod += __shfl_xor_sync(0xffffffffu, prod, o);
            }
            if (lane == 0)
            {
                red[r * (AC / 32) + warp] = prod;
            }
        }
    };

    if (!recur)
    {
        for (int i = 0; i < AR; i += RB)
        {
            double acc[RB];
            distances(xr, xc, i, j, d, rs, acc);
#pragma unroll
            for (int r = 0; r < RB; ++r)
            {
                emit(i + r, acc[r]);
            }
        }
    }
    else
    {
        // prologue: the first column of every warp, summed directly
        for (int q = threadIdx.x; q < AR * (AC / 32); q += AC)
        {
            const int w = q / AR, r = q % AR;
            bnd[r * (AC / 32) + w] = distance1(xr, xc, r, 32 * w, d, 1);
        }
        __syncthreads();
        double dprev = distance1(xr, xc, 0, j, d, 1);
        emit(0, dprev);
        const int jl = max(j - 1, 0);  // lane 0 takes bnd instead
        for (int r = 1; r < AR; ++r)
        {
            const double dleft = __shfl_up_sync(0xffffffffu, dprev, 1);
            const double z1 = __dsub_rn(xr[r - 1], xc[jl]);
            const double z2 = __dsub_rn(xr[r + d - 1], xc[j + d - 1]);
            const double rec = __dadd_rn(__dsub_rn(dleft, __dmul_rn(z1, z1)), __dmul_rn(z2, z2));
            const double dcur = (lane == 0) ? bnd[r * (AC / 32) + warp] : rec;
            emit(r, dcur);
            dprev = dcur;
        }
    }
    if (mean_partial != nullptr)
    {
        __syncthreads();
        for (int r = threadIdx.x; r < AR; r += AC)
        {
            int gi = i0 + r;
            if (gi < rows)
            {
                double s = 0.0;
#pragma unroll
                for (int w = 0; w < AC / 32; ++w)
                {
                    s += red[r * (AC / 32) + w];
                }
                mean_partial[static_cast<int64_t>(gi) * mean_parts + blockIdx.x] = s;
            }
        }
    }
}

__global__ void reduce_rows_kernel(const double *__restrict__ part, int m, int parts, double *__restrict__ out)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < m)
    {
        double s = 0.0;
        for (int q = 0; q < parts; ++q)
        {
            s += part[static_cast<int64_t>(r) * parts + q];
        }
        out[r] = s;
    }
}

size_t se_smem(int d, bool per_row)
{
    const size_t xr = per_row ? static_cast<size_t>(AR) * d : static_cast<size_t>(AR + d);
    return (xr + AC + d + 2 * AR * (AC / 32)) * sizeof(double);
}

template <int MODE, typename OutT>
void launch_se(const double *xrow, int rows, const double *xcol, int cols, int d, int T, const DeviceParams *p,
               OutT *out, int64_t ldo, const double *alpha, double *mean_partial, int parts, cudaStream_t s,
               const int64_t *row_offsets = nullptr, float *out32 = nullptr, int64_t ld32 = 0)
{
    if (rows <= 0 || cols <= 0)
    {
        return;
    }
    size_t smem = se_smem(d, row_offsets != nullptr);
    if (smem > 227 * 1024)
    {
        throw Error(1, "too many regressors for the assembly kernel");
    }
    if (smem > 48 * 1024)
    {
        ensure_smem_attr(reinterpret_cast<const void *>(se_kernel<MODE, OutT>), static_cast<int>(smem));
    }
    dim3 grid(ceil_div(cols, AC), ceil_div(rows, AR));
    se_kernel<MODE, OutT><<<grid, AC, smem, s>>>(xrow, rows, xcol, cols, d, T, p, out, ldo, alpha, mean_partial,
                                                 parts, row_offsets, out32, ld32);
    GPRAT_LAUNCH_CHECK();
}

}  // namespace

void assemble_covariance(const double *x, int n, int n_reg, int tile, const DeviceParams *p, double *K, int64_t ldk,
                         cudaStream_t s, float *K32, int64_t ld32)
{
    launch_se<0>(x, n, x, n, n_reg, tile, p, K, ldk, nullptr, nullptr, 0, s, nullptr, K32, ld32);
}

void assemble_cross(const double *xt, int m, const double *x, int n, int n_reg, const DeviceParams *p, double *Kx,
                    int64_t ldx, const double *alpha, double *mean_partial, int mean_parts, cudaStream_t s,
                    const int64_t *row_offsets)
{
    if (mean_partial != nullptr && mean_parts != ceil_div(n, AC))
    {
        throw Error(1, "assemble_cross: mean_parts must be ceil(n/128)");
    }
    launch_se<1>(xt, m, x, n, n_reg, 1, p, Kx, ldx, alpha, mean_partial, mean_parts, s, row_offsets);
}

void assemble_cross_f32(const double *xt, int m, const double *x, int n, int n_reg, const DeviceParams *p, float *Kx,
                        int64_t ldx, const double *alpha, double *mean_partial, int mean_parts, cudaStream_t s,
                        const int64_t *row_offsets)
{
    if (mean_partial != nullptr && mean_parts != ceil_div(n, AC))
    {
        throw Error(1, "assemble_cross: mean_parts must be ceil(n/128)");
    }
    launch_se<1>(xt, m, x, n, n_reg, 1, p, Kx, ldx, alpha, mean_partial, mean_parts, s, row_offsets);
}

void assemble_cross_dual(const double *xt, int m, const double *x, int n, int n_reg, const DeviceParams *p,
                         double *Kx, int64_t ldx, float *Kx32, int64_t ld32, cudaStream_t s)
{
    launch_se<1>(xt, m, x, n, n_reg, 1, p, Kx, ldx, nullptr, nullptr, 0, s, nullptr, Kx32, ld32);
}

namespace
{
// mean[r] = sum_c Kx[r][c] alpha[c]: one warp per row, 16-byte loads, a fixed
// summation order (deterministic).  HBM-bound: reads Kx once.
constexpr int MV_WARPS = 8;

__global__ void __launch_bounds__(32 * MV_WARPS) cross_mv_kernel(const double *__restrict__ Kx, int64_t ldx, int m,
                                                                 int n, const double *__restrict__ alpha,
                                                                 double *__restrict__ mean)
{
    const int r = blockIdx.x * MV_WARPS + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= m)
    {
        return;
    }
    const double *row = Kx + static_cast<int64_t>(r) * ldx;
    double s = 0.0;
    const int n2 = n & ~1;
    for (int c = 2 * lane; c < n2; c += 64)
    {
        const double2 k = *reinterpret_cast<const double2 *>(row + c);
        const double2 a = *reinterpret_cast<const double2 *>(alpha + c);
        s += k.x * a.x + k.y * a.y;
    }
    if ((n & 1) && lane == 0)
    {
        s += row[n - 1] * alpha[n - 1];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if (lane == 0)
    {
        mean[r] = s;
    }
}
}  // namespace

void cross_times_alpha(const double *Kx, int64_t ldx, int m, int n, const double *alpha, double *mean, cudaStream_t s)
{
    if (m <= 0)
    {
        return;
    }
    if ((ldx & 1) != 0 || (reinterpret_cast<uintptr_t>(Kx) & 15) != 0 || (reinterpret_cast<uintptr_t>(alpha) & 15) != 0)
    {
        throw Error(1, "cross_times_alpha: Kx and alpha must be 16-byte aligned with an even leading dimension");
    }
    cross_mv_kernel<<<ceil_div(m, MV_WARPS), 32 * MV_WARPS, 0, s>>>(Kx, ldx, m, n, alpha, mean);
    GPRAT_LAUNCH_CHECK();
}

void reduce_mean(const double *mean_partial, int m, int parts, double *mean, cudaStream_t s)
{
    if (m <= 0)
    {
        return;
    }
    reduce_rows_kernel<<<ceil_div(m, 256), 256, 0, s>>>(mean_partial, m, parts, mean);
    GPRAT_LAUNCH_CHECK();
}

void assemble_prior(const double *xt, int m, int n_reg, const DeviceParams *p, double *Kss, int64_t lds,
                    cudaStream_t s)
{
    launch_se<1>(xt, m, xt, m, n_reg, 1, p, Kss, lds, nullptr, nullptr, 0, s);
}

}  // namespace gprat_cu
