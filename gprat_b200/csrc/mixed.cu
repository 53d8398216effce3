// Mixed-precision pipeline (GPRAT_CU_PREC_MIXED_TF32 / _BF16).
//
// Factorisation (factor_mixed): K in FP64 and its FP32 working copy K32 in one
// pass; right-looking blocked Cholesky of
// K32 in outer panels of 1024 columns with a look-ahead of one panel, inside
// a panel left-looking over 128-column blocks:
//   - each 128 x 128 diagonal block is factored and inverted in FP64
//     (potrf_diag_f32), its FP64 diagonal kept for the log-determinant, its
//     inverse stored in FP32;
//   - panel solves P = P Linv^T and all updates run on the tcgen05 tensor
//     cores with TF32 operands (MIXED_TF32) or BF16 operands (MIXED_BF16, from
//     a BF16 copy of the factor), FP32 accumulation in TMEM.
// alpha (alpha_mixed): preconditioned conjugate gradients in FP64 on the
// exact FP64 K (a lower-storage symmetric mat-vec), preconditioned by the
// low-precision factor, to a relative residual of 1e-10.  The loss uses that
// alpha and the FP64 diagonal of the factor.
// Mean: the FP64 cross covariance with the refined alpha.
// Variance (variance_mixed, fit_predict_mixed): the cross covariance in FP32
// and the solve W L^T = K* on the tensor cores (recursive halving, or
// 512-column panels for few rows), row sums of W^2 accumulated in FP64.  Its
// error is that of the low-precision factor.
// fit_predict_mixed overlaps the variance solve with the factorisation and
// alpha's refinement on separate streams.
#include "gp_state.cuh"

#include <cmath>
#include <cstdlib>
#include <string>

namespace gprat_cu
{
namespace
{

// Iterations enqueued per solve.  Nothing waits on the host: once the
// residual test passes, the iterations after it return at once (their kernels
// read the converged flag), so the solve is one stream of launches that a
// CUDA graph can hold.  A solve that has not converged after these keeps its
// last iterate (4 iterations at n = 32768 with the TF32 preconditioner).
constexpr int PCG_ITERS = 24;
// 1e-10: four iterations at n = 32768 with a TF32 factor, the mean then within
// 1.5e-11 of the FP64 path's (a fifth iteration buys 3e-14)
constexpr double PCG_TOL = 1e-10;

// The relative residual PCG stops at: GPRAT_CU_PCG_TOL if it holds a number
// in [1e-15, 1e-6], else PCG_TOL (a tuning knob).
double pcg_tol()
{
    const char *v = std::getenv("GPRAT_CU_PCG_TOL");
    if (v != nullptr)
    {
        char *end = nullptr;
        const double t = std::strtod(v, &end);
        if (end != v && *end == '\0' && t >= 1e-15 && t <= 1e-6)
        {
            return t;
        }
    }
    return PCG_TOL;
}
constexpr int DOT_BLOCKS = 296;
constexpr int DOT_THREADS = 256;

struct MixedOps
{
    TcOperand L;     // K32 (TF32 view)
    TcOperand Lb;    // BF16 factor copy
    TcOperand Linv;  // Linv32 (TF32 view)
    bool bf16;
    const TcOperand &trail() const { return bf16 ? Lb : L; }
};

MixedOps make_ops(gprat_cu_gp *gp)
{
    MixedOps o;
    o.bf16 = gp->precision == GPRAT_CU_PREC_MIXED_BF16;
    tc_make_operand(o.L, gp->K32.ptr, gp->n, static_cast<int>(gp->ld32), gp->ld32, TcKind::TF32);
    tc_make_operand(o.Linv, gp->Linv32.ptr, gp->nblk * NB, NB, NB, TcKind::TF32);
    if (o.bf16)
    {
        tc_make_operand(o.Lb, gp->Lb.ptr, gp->n, static_cast<int>(gp->ld32), gp->ld32, TcKind::BF16);
    }
    return o;
}

TcGemmArgs tc_args(int M, int N, int K, int ar, int ac, int br, int bc, float *C, int64_t ldc, float alpha,
                   float beta, bool lower, double *rowsq, DeviceStatus *st)
{
    TcGemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.a_row0 = ar;
    g.a_col0 = ac;
    g.b_row0 = br;
    g.b_col0 = bc;
    g.C = C;
    g.ldc = ldc;
    g.alpha = alpha;
    g.beta = beta;
    g.lower = lower;
    g.rowsq = rowsq;
    g.rowsq_half = M;
    g.status = st;
    return g;
}

// ---------------------------------------------------------------------------
// FP64 symmetric mat-vec q = K p from the lower triangle (row-major, ld).
// One CTA per lower 128x128 tile (I, J <= I): it adds K_IJ p_J to the rows of
// block I and K_IJ^T p_I to the rows of block J.  Each (block, rows) pair of
// the partial buffer part[B][i] has exactly one writer, and q_i sums
// part[0..nblk)[i] in a fixed order, so the result is deterministic.
// Warp w reads rows 16w .. 16w+15 of the tile; lane l reads columns
// 4l .. 4l+3 of each row (two 16-byte loads, a warp reads a whole 1 KB row),
// all loads of eight rows issued before their arithmetic.  Row sums stay in
// registers (one per row) and are reduced across lanes once at the end,
// through shared memory; column sums are reduced across warps likewise.
constexpr int SV_THREADS = 256;

__global__ void __launch_bounds__(SV_THREADS) symv_tile_kernel(const double *__restrict__ K, int64_t ld, int n,
                                                               const double *__restrict__ p, double *__restrict__ part,
                                                               const int *skip)
{
    if (*skip != 0)
    {
        return;
    }
    __shared__ double pI[128], pJ[128];
    __shared__ double colsum[8][128];
    __shared__ double rowred[8][16][33];  // [warp][row][lane], padded against bank conflicts
    const int q = blockIdx.x;
    int I = static_cast<int>((sqrt(8.0 * q + 1.0) - 1.0) * 0.5);
    while ((I + 1) * (I + 2) / 2 <= q)
    {
        ++I;
    }
    while (I > 0 && I * (I + 1) / 2 > q)
    {
        --I;
    }
    const int J = q - I * (I + 1) / 2;
    const int i0 = I * 128, j0 = J * 128;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = threadIdx.x; t < 128; t += SV_THREADS)
    {
        pI[t] = (i0 + t < n) ? p[i0 + t] : 0.0;
        pJ[t] = (j0 + t < n) ? p[j0 + t] : 0.0;
    }
    __syncthreads();
    const int c0 = 4 * lane;  // this lane's first column in the tile
    double pj[4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
    {
        pj[c] = pJ[c0 + c];
    }
    const bool full = (I != J) && (i0 + 128 <= n) && (j0 + 128 <= n);
    double rs[16];
    double cs[4] = { 0.0, 0.0, 0.0, 0.0 };
#pragma unroll
    for (int h = 0; h < 2; ++h)
    {
        double2 v[8][2];
#pragma unroll
        for (int k = 0; k < 8; ++k)
        {
            const int r = 16 * warp + 8 * h + k;
            const int gi = min(i0 + r, n - 1);
            const double2 *src = reinterpret_cast<const double2 *>(K + static_cast<int64_t>(gi) * ld + j0 + c0);
            if (full || (i0 + r < n && j0 + c0 + 3 < n))
            {
                v[k][0] = src[0];
                v[k][1] = src[1];
            }
            else
            {
                // ragged edge: element loads inside the matrix, zero outside
                double e[4];
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    e[c] = (i0 + r < n && j0 + c0 + c < n) ? K[static_cast<int64_t>(gi) * ld + j0 + c0 + c] : 0.0;
                }
                v[k][0] = make_double2(e[0], e[1]);
                v[k][1] = make_double2(e[2], e[3]);
            }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
        {
            const int r = 16 * warp + 8 * h + k;
            double e[4] = { v[k][0].x, v[k][0].y, v[k][1].x, v[k][1].y };
            if (!full)
            {
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    // diagonal tile: the lower triangle only (the diagonal once)
                    e[c] = (I == J && c0 + c > r) ? 0.0 : e[c];
                }
            }
            double sr = 0.0;
            const double pir = pI[r];
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                sr += e[c] * pj[c];
                // transposed part: strictly below the diagonal on a diagonal tile
                cs[c] += ((I == J && c0 + c == r) ? 0.0 : e[c]) * pir;
            }
            rs[8 * h + k] = sr;
        }
    }
#pragma unroll
    for (int k = 0; k < 16; ++k)
    {
        rowred[warp][k][lane] = rs[k];
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
    {
        colsum[warp][c0 + c] = cs[c];
    }
    __syncthreads();
    // row r of the tile: warp r / 16, row slot r % 16; two threads per row
    // each sum 16 lanes, then combine
    {
        const int r = threadIdx.x >> 1, half = threadIdx.x & 1;
        const double *src = &rowred[r >> 4][r & 15][16 * half];
        double sr = 0.0;
#pragma unroll
        for (int l = 0; l < 16; ++l)
        {
            sr += src[l];
        }
        sr += __shfl_xor_sync(0xffffffffu, sr, 1);
        if (half == 0)
        {
            double c = 0.0;
#pragma unroll
            for (int w = 0; w < SV_THREADS / 32; ++w)
            {
                c += colsum[w][r];
            }
            if (I == J)
            {
                if (i0 + r < n)
                {
                    part[static_cast<int64_t>(I) * n + i0 + r] = sr + c;
                }
            }
            else
            {
                if (i0 + r < n)
                {
                    part[static_cast<int64_t>(J) * n + i0 + r] = sr;
                }
                if (j0 + r < n)
                {
                    part[static_cast<int64_t>(I) * n + j0 + r] = c;
                }
            }
        }
    }
}

__global__ void symv_reduce_kernel(const double *__restrict__ part, int nblk, int n, double *__restrict__ q,
                                   const int *skip)
{
    if (*skip != 0)
    {
        return;
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        double s = 0.0;
        for (int b = 0; b < nblk; ++b)
        {
            s += part[static_cast<int64_t>(b) * n + i];
        }
        q[i] = s;
    }
}

// ---------------------------------------------------------------------------
// PCG helpers (all scalars live in PcgScalars on the device)

__global__ void __launch_bounds__(DOT_THREADS) dot_partial_kernel(const double *__restrict__ a,
                                                                  const double *__restrict__ b, int n,
                                                                  double *__restrict__ part, const int *skip)
{
    if (skip != nullptr && *skip != 0)
    {
        return;
    }
    __shared__ double red[DOT_THREADS];
    double s = 0.0;
    for (int i = blockIdx.x * DOT_THREADS + threadIdx.x; i < n; i += DOT_BLOCKS * DOT_THREADS)
    {
        s += a[i] * b[i];
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = DOT_THREADS / 2; w > 0; w >>= 1)
    {
        if (threadIdx.x < w)
        {
            red[threadIdx.x] += red[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        part[blockIdx.x] = red[0];
    }
}

__device__ double sum_parts(const double *part)
{
    double s = 0.0;
    for (int b = 0; b < DOT_BLOCKS; ++b)
    {
        s += part[b];
    }
    return s;
}

// which: 0 = yy (init), 1 = rz (init), 2 = pq -> a, 3 = rr -> converged, 4 = rz -> b
__global__ void pcg_scalar_kernel(PcgScalars *s, const double *part, int which, double tol)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
    {
        return;
    }
    if (which >= 2 && s->converged != 0)
    {
        return;  // an iteration after convergence: nothing changes
    }
    const double v = sum_parts(part);
    switch (which)
    {
        case 0:
            s->yy = v;
            s->converged = (v == 0.0) ? 1 : 0;
            s->iters = 0;
            break;
        case 1: s->rz = v; break;
        case 2:
            s->pq = v;
            s->a = (v != 0.0) ? s->rz / v : 0.0;
            break;
        case 3:
            s->rr = v;
            s->iters += 1;
            s->converged = (v <= tol * tol * s->yy) ? 1 : 0;
            break;
        case 4:
            s->b = (s->rz != 0.0) ? v / s->rz : 0.0;
            s->rz = v;
            break;
    }
}

// x += a p; r -= a q
__global__ void pcg_update_kernel(const PcgScalars *__restrict__ s, double *__restrict__ x,
                                  double *__restrict__ r, const double *__restrict__ p,
                                  const double *__restrict__ q, int n)
{
    if (s->converged != 0)
    {
        return;
    }
    const double a = s->a;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        x[i] += a * p[i];
        r[i] -= a * q[i];
    }
}

// p = z + b p
__global__ void pcg_direction_kernel(const PcgScalars *__restrict__ s, double *__restrict__ p,
                                     const double *__restrict__ z, int n)
{
    if (s->converged != 0)
    {
        return;
    }
    const double b = s->b;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        p[i] = z[i] + b * p[i];
    }
}

// skip (optional, device): the product is not needed when *skip != 0
void dot(const double *a, const double *b, int n, double *part, cudaStream_t s, const int *skip = nullptr)
{
    dot_partial_kernel<<<DOT_BLOCKS, DOT_THREADS, 0, s>>>(a, b, n, part, skip);
    GPRAT_LAUNCH_CHECK();
}

void scalar(PcgScalars *ps, const double *part, int which, cudaStream_t s)
{
    pcg_scalar_kernel<<<1, 32, 0, s>>>(ps, part, which, pcg_tol());
    GPRAT_LAUNCH_CHECK();
}

int blocks_for(int n) { return std::min(ceil_div(n, 256), 148 * 8); }

void symv(gprat_cu_gp *gp, const double *p, double *q, cudaStream_t s, const int *skip)
{
    const int tiles = gp->nblk * (gp->nblk + 1) / 2;
    symv_tile_kernel<<<tiles, SV_THREADS, 0, s>>>(gp->K.ptr, gp->ld, gp->n, p, gp->symv_part.ptr, skip);
    GPRAT_LAUNCH_CHECK();
    symv_reduce_kernel<<<ceil_div(gp->n, 256), 256, 0, s>>>(gp->symv_part.ptr, gp->nblk, gp->n, q, skip);
    GPRAT_LAUNCH_CHECK();
}

// z = (L L^T)^-1 r with the low-precision factor; solve_ctas > 0 bounds the
// solves' grids; nothing is solved when *skip != 0.
void precondition(gprat_cu_gp *gp, const double *r, double *z, cudaStream_t s, int solve_ctas, const int *skip)
{
    GPRAT_CUDA_CHECK(cudaMemcpyAsync(z, r, gp->n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    gp->flags.ensure(2);
    gp->trsv_b.ensure(gp->n);
    trsv_fused_forward_f32(gp->K32.ptr, gp->ld32, gp->Linv32.ptr, gp->n, z, gp->flags.ptr, gp->trsv_b.ptr,
                           gp->status.ptr, s, solve_ctas, skip);
    trsv_fused_backward_f32(gp->K32.ptr, gp->ld32, gp->Linv32.ptr, gp->n, z, gp->flags.ptr, gp->trsv_b.ptr,
                            gp->status.ptr, s, solve_ctas, skip);
}

}  // namespace

// Helpers shared with the int8-emulated FP64 pipeline (ozaki_path.cu).

// Share of the SMs the main stream's trailing update may hold while the
// look-ahead stream works next to it (persistent CTAs never yield their SM,
// so the side stream, which carries the critical path, needs SMs left free).
#ifndef GPRAT_LOOKAHEAD_MAIN_PERCENT
#define GPRAT_LOOKAHEAD_MAIN_PERCENT 70
#endif
#ifndef GPRAT_MIXED_PANEL_BLOCKS
#define GPRAT_MIXED_PANEL_BLOCKS 8  // outer panels of 8 x 128 columns
#endif
#ifndef GPRAT_LOOKAHEAD_MAIN_PERCENT_LARGE
#define GPRAT_LOOKAHEAD_MAIN_PERCENT_LARGE 70
#endif
#ifndef GPRAT_LOOKAHEAD_LARGE_ROWS
#define GPRAT_LOOKAHEAD_LARGE_ROWS 16384
#endif

// A tuning knob: the environment variable `name` if it holds an integer in
// [lo, hi], else the compiled default.
int knob(const char *name, int dflt, int lo, int hi)
{
    const char *v = std::getenv(name);
    if (v != nullptr)
    {
        char *end = nullptr;
        const long p = std::strtol(v, &end, 10);
        if (end != v && *end == '\0' && p >= lo && p <= hi)
        {
            return static_cast<int>(p);
        }
    }
    return dflt;
}

// A share of the SMs in percent (knob in [10, 100]).
int sm_percent(const char *name, int dflt) { return knob(name, dflt, 10, 100); }

void ensure_lookahead(gprat_cu_gp *gp, int nevents)
{
    if (gp->side == nullptr)
    {
        int least = 0, greatest = 0;
        GPRAT_CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        GPRAT_CUDA_CHECK(cudaStreamCreateWithPriority(&gp->side, cudaStreamNonBlocking, greatest));
        GPRAT_CUDA_CHECK(cudaStreamCreateWithPriority(&gp->vstream, cudaStreamNonBlocking, least));
    }
    while (static_cast<int>(gp->events.size()) < nevents)
    {
        cudaEvent_t e = nullptr;
        GPRAT_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        gp->events.push_back(e);
    }
}

// Events of one factorisation (two per outer panel of at least one block,
// one to start) and seven for fit_predict_mixed, at the end.
// the look-ahead's 2 per block column and 1, the pipelines' 7 named ones and
// up to 8 split points of the int8 path's early variance solve
int lookahead_events(int n) { return 2 * ceil_div(n, NB) + 16; }

TcGemmArgs limited(TcGemmArgs a, int max_ctas)
{
    a.max_ctas = max_ctas;
    return a;
}

// Right-looking Cholesky of the FP32 working copy in outer panels of nbo
// columns (inner blocks of NB), with a look-ahead of one panel:
//   side stream (high priority): factor panel k (diagonal blocks in FP64,
//     panel solves and the in-panel updates on tcgen05), then apply panel k
//     to the columns of panel k+1 and factor panel k+1;
//   main stream: the trailing update of everything right of panel k+1 with
//     panel k (the bulk of the flops), on GPRAT_LOOKAHEAD_MAIN_PERCENT % of the SMs while the
//     side stream works next to it (the panel chain is the critical path).
// Events order the two streams: panel k+1's columns are written by the
// update of panel k-1 (main) before the side stream touches them, and the
// update of panel k waits for panel k's factorisation.
// splits (optional): (c, e) pairs; e is recorded on the side stream once
// columns [0, c) of the factor are final (all rows), so that work which needs
// only those columns can start before the factorisation ends.
void factor_mixed(gprat_cu_gp *gp, cudaStream_t s, const std::vector<std::pair<int, cudaEvent_t>> &splits)
{
    const int n = gp->n;
    if (n % NB != 0)
    {
        throw Error(GPRAT_CU_ERR_INVALID_ARG,
                    "mixed precision needs n_tiles * n_tile_size to be a multiple of 128 (got " + std::to_string(n) +
                        ")");
    }
    const int64_t ld32 = gp->ld32;
    gp->K32.ensure(static_cast<int64_t>(n) * ld32);
    gp->Linv32.ensure(static_cast<int64_t>(gp->nblk) * NB * NB);
    gp->D64.ensure(static_cast<int64_t>(NB) * NB + n);  // one block + the FP64 diagonal of L
    if (gp->precision == GPRAT_CU_PREC_MIXED_BF16)
    {
        gp->Lb.ensure(static_cast<int64_t>(n) * ld32);
    }
    double *ldiag = gp->D64.ptr + NB * NB;
    // outer panel width (a multiple of the 128-wide diagonal blocks)
    const int nbo = NB * knob("GPRAT_CU_MIXED_PANEL_BLOCKS", GPRAT_MIXED_PANEL_BLOCKS, 1, 16);
    const int nout = ceil_div(n, nbo);
    ensure_lookahead(gp, lookahead_events(n));
    cudaStream_t side = gp->side;
    auto evF = [&](int k) { return gp->events[1 + k]; };
    auto evR = [&](int k) { return gp->events[1 + nout + k]; };
    const int sms = device_sm_count();
    // While the trailing matrix is large the update of panel k outlasts the
    // panel chain by far, so it may take a larger share of the SMs.
    const int main_percent = sm_percent("GPRAT_CU_LOOKAHEAD_MAIN_PERCENT", GPRAT_LOOKAHEAD_MAIN_PERCENT);
    const int main_percent_large = sm_percent("GPRAT_CU_LOOKAHEAD_MAIN_PERCENT_LARGE", GPRAT_LOOKAHEAD_MAIN_PERCENT_LARGE);
    const int large_rows = knob("GPRAT_CU_LOOKAHEAD_LARGE_ROWS", GPRAT_LOOKAHEAD_LARGE_ROWS, 0, 1 << 30);

    {
        StepScope step("assembly", s);
        assemble_covariance(gp->x.ptr, n, gp->d, gp->T, gp->params.ptr, gp->K.ptr, gp->ld, s, gp->K32.ptr, ld32);
    }
    StepScope step("cholesky", s);
    GPRAT_CUDA_CHECK(cudaEventRecord(gp->events[0], s));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(side, gp->events[0], 0));
    const MixedOps ops = make_ops(gp);
    float *K32 = gp->K32.ptr;
    auto at = [&](int r, int c) { return K32 + static_cast<int64_t>(r) * ld32 + c; };

    // factor panel [K0, pend): diagonal blocks, panel solves, in-panel updates.
    // Left-looking inside the panel (the default): before block column r0 is
    // factored it receives the updates of every solved block column of the
    // panel left of it in one GEMM of depth r0 - K0 (n - r0 rows, 128
    // columns).  Right-looking: each solved block column updates all the
    // panel's columns right of it at once; the same flops in twice the tiles.
    const bool left = knob("GPRAT_CU_PANEL_LEFT_LOOKING", 1, 0, 1) != 0;
    auto factor_panel = [&](int K0, int pend, int ctas)
    {
        for (int r0 = K0; r0 < pend; r0 += NB)
        {
            const int k = r0 / NB;
            if (left && r0 > K0)
            {
                tc_gemm(ops.trail(), ops.trail(),
                        limited(tc_args(n - r0, NB, r0 - K0, r0, K0, r0, K0, at(r0, r0), ld32, -1.0f, 1.0f, false,
                                        nullptr, gp->status.ptr),
                                ctas),
                        side);
            }
            // the diagonal block of L in the working copy and an FP64 inverse
            // are not used downstream (solves use Linv32, the log-determinant
            // the FP64 diagonal): neither is written
            potrf_diag_f32(at(r0, r0), ld32, NB, r0, nullptr, 0, gp->Linv32.ptr + static_cast<int64_t>(k) * NB * NB,
                           NB, ldiag + r0, gp->status.ptr, side, false);
            const int rows = n - r0 - NB;
            if (rows > 0)
            {
                // panel solve P = P Linv^T on the tensor cores (TF32), in place
                tc_gemm(ops.L, ops.Linv,
                        limited(tc_args(rows, NB, NB, r0 + NB, r0, k * NB, 0, at(r0 + NB, r0), ld32, 1.0f, 0.0f, false,
                                        nullptr, gp->status.ptr),
                                ctas),
                        side);
            }
            if (ops.bf16)
            {
                convert_f32_to_bf16(at(r0, r0), ld32, gp->Lb.ptr + static_cast<int64_t>(r0) * ld32 + r0, ld32,
                                    n - r0, NB, side);
            }
            // the rest of the panel's columns, every row below the block, in one
            // launch (the strict upper triangle of the working copy is scratch:
            // nothing reads it, so its in-panel part is updated too)
            const int ncols = pend - (r0 + NB);
            if (!left && ncols > 0)
            {
                tc_gemm(ops.trail(), ops.trail(),
                        limited(tc_args(n - (r0 + NB), ncols, NB, r0 + NB, r0, r0 + NB, r0, at(r0 + NB, r0 + NB), ld32,
                                        -1.0f, 1.0f, false, nullptr, gp->status.ptr),
                                ctas),
                        side);
            }
        }
    };

    size_t next_split = 0;  // splits are in ascending column order
    auto maybe_split = [&](int done_cols)
    {
        while (next_split < splits.size() && done_cols >= splits[next_split].first)
        {
            GPRAT_CUDA_CHECK(cudaEventRecord(splits[next_split].second, side));
            ++next_split;
        }
    };
    factor_panel(0, std::min(nbo, n), 0);
    maybe_split(std::min(nbo, n));
    GPRAT_CUDA_CHECK(cudaEventRecord(evF(0), side));
    for (int k = 0; k < nout; ++k)
    {
        const int K0 = k * nbo;
        const int pend = std::min(K0 + nbo, n);
        const int bo = pend - K0;
        const int next_end = std::min(pend + nbo, n);  // end of panel k+1
        const int rest = n - next_end;
        const bool ahead = k + 1 < nout;
        // main: everything right of panel k+1, with panel k
        GPRAT_CUDA_CHECK(cudaStreamWaitEvent(s, evF(k), 0));
        if (rest > 0)
        {
            tc_gemm(ops.trail(), ops.trail(),
                    limited(tc_args(rest, rest, bo, next_end, K0, next_end, K0, at(next_end, next_end), ld32, -1.0f,
                                    1.0f, true, nullptr, gp->status.ptr),
                            ahead ? std::max(1, sms * (rest >= large_rows ? main_percent_large : main_percent) / 100)
                                  : 0),
                    s);
        }
        GPRAT_CUDA_CHECK(cudaEventRecord(evR(k), s));
        if (!ahead)
        {
            break;
        }
        // side: panel k applied to panel k+1's columns, then panel k+1 factored
        const int side_ctas = 0;  // the critical path takes every SM it can get
        if (k >= 1)
        {
            GPRAT_CUDA_CHECK(cudaStreamWaitEvent(side, evR(k - 1), 0));
        }
        // panel k+1's columns, every row from its diagonal down, in one launch
        // (the upper triangle of its diagonal region is scratch)
        const int nb = next_end - pend;
        tc_gemm(ops.trail(), ops.trail(),
                limited(tc_args(n - pend, nb, bo, pend, K0, pend, K0, at(pend, pend), ld32, -1.0f, 1.0f, false,
                                nullptr, gp->status.ptr),
                        side_ctas),
                side);
        factor_panel(pend, next_end, side_ctas);
        maybe_split(next_end);
        GPRAT_CUDA_CHECK(cudaEventRecord(evF(k + 1), side));
    }
}

void alpha_mixed(gprat_cu_gp *gp, cudaStream_t s, int solve_ctas)
{
    const int n = gp->n;
    for (DevBuf<double> *b : { &gp->pcg_r, &gp->pcg_z, &gp->pcg_p, &gp->pcg_q })
    {
        b->ensure(n);
    }
    gp->symv_part.ensure(static_cast<int64_t>(gp->nblk) * n + 3 * DOT_BLOCKS);
    gp->pcg_s.ensure(1);
    double *part = gp->symv_part.ptr + static_cast<int64_t>(gp->nblk) * n;  // dot partials
    PcgScalars *ps = gp->pcg_s.ptr;
    double *x = gp->alpha.ptr, *r = gp->pcg_r.ptr, *z = gp->pcg_z.ptr, *p = gp->pcg_p.ptr, *q = gp->pcg_q.ptr;
    const int nb = blocks_for(n);

    const int *done = &ps->converged;  // device flag, set by the residual test
    GPRAT_CUDA_CHECK(cudaMemsetAsync(x, 0, n * sizeof(double), s));
    GPRAT_CUDA_CHECK(cudaMemcpyAsync(r, gp->y.ptr, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    dot(r, r, n, part, s);
    scalar(ps, part, 0, s);
    precondition(gp, r, z, s, solve_ctas, done);
    dot(r, z, n, part, s, done);
    scalar(ps, part, 1, s);
    GPRAT_CUDA_CHECK(cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    for (int it = 0; it < PCG_ITERS; ++it)
    {
        symv(gp, p, q, s, done);
        dot(p, q, n, part, s, done);
        scalar(ps, part, 2, s);
        pcg_update_kernel<<<nb, 256, 0, s>>>(ps, x, r, p, q, n);
        GPRAT_LAUNCH_CHECK();
        dot(r, r, n, part, s, done);
        scalar(ps, part, 3, s);
        precondition(gp, r, z, s, solve_ctas, done);
        dot(r, z, n, part, s, done);
        scalar(ps, part, 4, s);
        pcg_direction_kernel<<<nb, 256, 0, s>>>(ps, p, z, n);
        GPRAT_LAUNCH_CHECK();
    }
}

void loss_mixed(gprat_cu_gp *gp, cudaStream_t s)
{
    // y . alpha with the refined alpha, log-determinant from the FP64 diagonal
    loss_kernel(gp->y.ptr, gp->alpha.ptr, gp->D64.ptr + NB * NB, 0, gp->n, gp->params.ptr, s);
}

namespace
{

// Below this many test rows the variance solve runs in 512-column panels
// (short GEMMs over many CTAs), at or above it by recursive halving (deep
// GEMMs; W is read and written once per level instead of once per panel).
constexpr int RECURSIVE_MIN_ROWS = 2048;

// Operands and buffers of one variance solve W L^T = K* (in place in W).
struct VarianceSolve
{
    gprat_cu_gp *gp;
    MixedOps ops;
    TcOperand opW;   // W (TF32 view)
    TcOperand opWb;  // BF16 copy of the solved columns of W (MIXED_BF16)
    float *W;
    int64_t ld32;
    int m;
    int max_ctas;
    cudaStream_t s;

    const TcOperand &wt() const { return ops.bf16 ? opWb : opW; }

    // W[:, c0:c0+128) := W[:, c0:c0+128) Linv_k^T (k = c0 / 128), row sums of
    // squares into vacc.
    void leaf(int c0) const
    {
        const int k = c0 / NB;
        tc_gemm(opW, ops.Linv,
                limited(tc_args(m, NB, NB, 0, c0, k * NB, 0, W + c0, ld32, 1.0f, 0.0f, false, gp->vacc.ptr,
                                gp->status.ptr),
                        max_ctas),
                s);
        if (ops.bf16)
        {
            convert_f32_to_bf16(W + c0, ld32, gp->Wb.ptr + c0, ld32, m, NB, s);
        }
    }

    // W[:, cols) -= W[:, k0:k1) L[cols, k0:k1)^T
    void update(int k0, int k1, int c0, int c1) const
    {
        if (k1 <= k0 || c1 <= c0)
        {
            return;
        }
        tc_gemm(wt(), ops.trail(),
                limited(tc_args(m, c1 - c0, k1 - k0, 0, k0, c0, k0, W + c0, ld32, -1.0f, 1.0f, false, nullptr,
                                gp->status.ptr),
                        max_ctas),
                s);
    }

    // Right-looking in panels of 512 columns (inner blocks of 128): every
    // update has depth 128 or 512, so each GEMM is short.  For few rows (a
    // single row of tiles) this keeps many CTAs busy and no SM is held for
    // long, where the recursive solve would run depth-16384 updates on a
    // few CTAs.
    void solve_panels(int n) const
    {
        for (int K0 = 0; K0 < n; K0 += NBO)
        {
            const int pend = std::min(K0 + NBO, n);
            for (int c0 = K0; c0 < pend; c0 += NB)
            {
                leaf(c0);
                if (c0 + NB < pend)
                {
                    update(c0, c0 + NB, c0 + NB, pend);
                }
            }
            if (pend < n)
            {
                update(K0, pend, pend, n);
            }
        }
    }

    // W[:, c0:c1) := W[:, c0:c1) L[c0:c1, c0:c1)^-T, for columns that already
    // hold every update from the columns left of c0.  Recursive halving: the
    // update between the halves is one GEMM of depth (mid - c0), so each
    // level of the recursion reads and writes W once (the K = 512 outer
    // panels of the factorisation would read and write it n / 512 times).
    void solve(int c0, int c1) const
    {
        if (c1 <= c0)
        {
            return;  // an empty range (a split of a factor with fewer than four blocks)
        }
        if (c1 - c0 <= NB)
        {
            leaf(c0);
            return;
        }
        const int mid = c0 + ((c1 - c0) / NB / 2) * NB;
        solve(c0, mid);
        update(c0, mid, mid, c1);
        solve(mid, c1);
    }
};

}  // namespace

// Mean (when d_mean != nullptr, from the refined alpha) and variance (when
// d_var != nullptr) for m test points.  max_ctas bounds the grid of the
// variance solve's GEMMs (0: every SM), so that another stream can run next
// to it.  recursive: the variance solve may use recursive halving (for
// RECURSIVE_MIN_ROWS rows or more); its deepest GEMMs hold every SM for
// milliseconds, so callers that share the GPU with latency-sensitive work
// (a serving batch) keep to the panel order, whose GEMMs are short.
void variance_mixed(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s,
                    const int64_t *row_offsets, int max_ctas, bool recursive)
{
    const int n = gp->n;
    const int64_t ld32 = gp->ld32;
    const int parts = ceil_div(n, 128);
    gp->mean_part.ensure(static_cast<int64_t>(m) * parts);
    gp->W32.ensure(static_cast<int64_t>(m) * ld32);
    gp->vacc.ensure(2 * static_cast<int64_t>(m));  // one accumulator per column half of the GEMM tile
    const bool bf16 = gp->precision == GPRAT_CU_PREC_MIXED_BF16;
    if (bf16)
    {
        gp->Wb.ensure(static_cast<int64_t>(m) * ld32);
    }
    float *W = gp->W32.ptr;
    {
        StepScope step("prediction", s);
        assemble_cross_f32(d_xt, m, gp->x.ptr, n, gp->d, gp->params.ptr, W, ld32,
                           d_mean != nullptr ? gp->alpha.ptr : nullptr,
                           d_mean != nullptr ? gp->mean_part.ptr : nullptr, parts, s, row_offsets);
        if (d_mean != nullptr)
        {
            reduce_mean(gp->mean_part.ptr, m, parts, d_mean, s);
        }
    }
    if (d_var == nullptr)
    {
        return;
    }
    StepScope step("forward KcK", s);
    GPRAT_CUDA_CHECK(cudaMemsetAsync(gp->vacc.ptr, 0, 2 * m * sizeof(double), s));
    VarianceSolve v{ gp, make_ops(gp), {}, {}, W, ld32, m, max_ctas, s };
    tc_make_operand(v.opW, W, m, static_cast<int>(ld32), ld32, TcKind::TF32);
    if (bf16)
    {
        tc_make_operand(v.opWb, gp->Wb.ptr, m, static_cast<int>(ld32), ld32, TcKind::BF16);
    }
    if (recursive && m >= RECURSIVE_MIN_ROWS)
    {
        v.solve(0, n);
    }
    else
    {
        v.solve_panels(n);
    }
    finalize_variance(gp->vacc.ptr, m, gp->params.ptr, d_var, s, gp->vacc.ptr + m);
}

// Share of the SMs the variance solve's GEMMs hold while alpha is refined
// next to them (the refinement's solves are latency-bound and need few SMs),
// and the grid of those solves (0: one CTA per row block).
#ifndef GPRAT_SOLVE_CTAS
#define GPRAT_SOLVE_CTAS 0
#endif
#ifndef GPRAT_VARIANCE_PERCENT
#define GPRAT_VARIANCE_PERCENT 75
#endif
#ifndef GPRAT_VARIANCE_EARLY_PERCENT
#define GPRAT_VARIANCE_EARLY_PERCENT 70
#endif

// Fit, mean and variance (predict_with_uncertainty).
//   caller's stream `s` + high-priority side stream: the factorisation;
//   low-priority variance stream: the cross covariance K* (independent of the
//     factor) from the start; with RECURSIVE_MIN_ROWS test rows or more, the
//     first half of the recursive variance solve (its left half and the big
//     update of the right half) as soon as the factor's left half is final,
//     and the next quarter once three quarters are, beside the
//     factorisation's second half (whose panel chain leaves SMs idle), on
//     GPRAT_VARIANCE_EARLY_PERCENT % of the SMs; the rest once the factor is
//     complete, on GPRAT_VARIANCE_PERCENT %;
//   side stream, after the factorisation: alpha's refinement (FP64 PCG) and
//     the mean (from K* kept in FP64 by the variance stream's assembly).
// `s` waits for both at the end.
void fit_predict_mixed(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s)
{
    const int n = gp->n;
    const int ne = lookahead_events(n);
    ensure_lookahead(gp, ne);
    cudaEvent_t kx_ready = gp->events[ne - 7];
    cudaEvent_t begin = gp->events[ne - 6], half = gp->events[ne - 5], three_q = gp->events[ne - 4];
    cudaEvent_t factored = gp->events[ne - 3], refined = gp->events[ne - 2], solved = gp->events[ne - 1];
    cudaStream_t side = gp->side, vs = gp->vstream;
    const int sms = device_sm_count();
    const int parts = ceil_div(n, 128);
    const bool early = m >= RECURSIVE_MIN_ROWS;
    const int h = (n / NB / 2) * NB;                      // the recursive solve's first split
    const int h2 = h + ((n - h) / NB / 2) * NB;           // and the split of its right half
    // buffers first (an allocation must not fall between launches of different streams)
    gp->mean_part.ensure(static_cast<int64_t>(std::max(m, 1)) * parts);
    gp->W32.ensure(static_cast<int64_t>(std::max(m, 1)) * gp->ld32);
    gp->vacc.ensure(2 * static_cast<int64_t>(std::max(m, 1)));
    if (early)
    {
        gp->W.ensure(static_cast<int64_t>(m) * gp->ld);  // K* in FP64, for the mean
    }
    if (gp->precision == GPRAT_CU_PREC_MIXED_BF16)
    {
        gp->Wb.ensure(static_cast<int64_t>(std::max(m, 1)) * gp->ld32);
    }
    GPRAT_CUDA_CHECK(cudaEventRecord(begin, s));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(vs, begin, 0));
    std::vector<std::pair<int, cudaEvent_t>> splits;
    // GPRAT_CU_VARIANCE_SPLITS: 1 starts only the first half early, 2 (default) also the next quarter
    const bool two = knob("GPRAT_CU_VARIANCE_SPLITS", 2, 1, 2) == 2;
    if (early)
    {
        splits = { { h, half }, { two ? h2 : n + 1, three_q } };
    }
    factor_mixed(gp, s, splits);
    GPRAT_CUDA_CHECK(cudaEventRecord(factored, s));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(side, factored, 0));
    if (m > 0)
    {
        const int late_ctas =
            std::max(1, sms * sm_percent("GPRAT_CU_VARIANCE_PERCENT", GPRAT_VARIANCE_PERCENT) / 100);
        if (early)
        {
            float *W = gp->W32.ptr;
            const int64_t ld32 = gp->ld32;
            {
                // K* once, in FP64 (kept for the mean: a mat-vec with alpha
                // once alpha is refined, instead of a second assembly) and FP32
                StepScope step("prediction", vs);
                assemble_cross_dual(d_xt, m, gp->x.ptr, n, gp->d, gp->params.ptr, gp->W.ptr, gp->ld, W, ld32, vs);
                GPRAT_CUDA_CHECK(cudaEventRecord(kx_ready, vs));
            }
            StepScope step("forward KcK", vs);
            GPRAT_CUDA_CHECK(cudaMemsetAsync(gp->vacc.ptr, 0, 2 * m * sizeof(double), vs));
            VarianceSolve v{ gp, make_ops(gp), {}, {}, W, ld32, m, 0, vs };
            tc_make_operand(v.opW, W, m, static_cast<int>(ld32), ld32, TcKind::TF32);
            if (gp->precision == GPRAT_CU_PREC_MIXED_BF16)
            {
                tc_make_operand(v.opWb, gp->Wb.ptr, m, static_cast<int>(ld32), ld32, TcKind::BF16);
            }
            GPRAT_CUDA_CHECK(cudaStreamWaitEvent(vs, half, 0));
            v.max_ctas = std::max(
                1, sms * sm_percent("GPRAT_CU_VARIANCE_EARLY_PERCENT", GPRAT_VARIANCE_EARLY_PERCENT) / 100);
            v.solve(0, h);
            v.update(0, h, h, n);
            GPRAT_CUDA_CHECK(cudaStreamWaitEvent(vs, three_q, 0));
            v.solve(h, h2);
            v.update(h, h2, h2, n);
            GPRAT_CUDA_CHECK(cudaStreamWaitEvent(vs, factored, 0));
            v.max_ctas = late_ctas;
            v.solve(h2, n);
            finalize_variance(gp->vacc.ptr, m, gp->params.ptr, d_var, vs, gp->vacc.ptr + m);
        }
        else
        {
            GPRAT_CUDA_CHECK(cudaStreamWaitEvent(vs, factored, 0));
            variance_mixed(gp, d_xt, m, nullptr, d_var, vs, nullptr, late_ctas);
        }
    }
    GPRAT_CUDA_CHECK(cudaEventRecord(solved, vs));
    {
        StepScope step("alpha refinement", side);
        alpha_mixed(gp, side, knob("GPRAT_CU_SOLVE_CTAS", GPRAT_SOLVE_CTAS, 0, 100000));
    }
    if (m > 0)
    {
        StepScope step("prediction", side);
        if (early)
        {
            GPRAT_CUDA_CHECK(cudaStreamWaitEvent(side, kx_ready, 0));
            cross_times_alpha(gp->W.ptr, gp->ld, m, n, gp->alpha.ptr, d_mean, side);
        }
        else
        {
            assemble_cross(d_xt, m, gp->x.ptr, n, gp->d, gp->params.ptr, nullptr, 0, gp->alpha.ptr,
                           gp->mean_part.ptr, parts, side, nullptr);
            reduce_mean(gp->mean_part.ptr, m, parts, d_mean, side);
        }
    }
    GPRAT_CUDA_CHECK(cudaEventRecord(refined, side));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(s, refined, 0));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(s, solved, 0));
}

}  // namespace gprat_cu
