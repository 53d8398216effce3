// The FP64-accurate pipeline on the int8 tensor cores (GPRAT_CU_PREC_FP64_INT8).
//
// The factorisation and the solves keep FP64 data: K is factored in place as
// in the FP64 path and every matrix product -- in-panel and trailing
// updates, panel solves with the diagonal-block inverses, and every product
// of the variance solve W L^T = K* -- runs as an int8-emulated FP64 GEMM
// (oz_gemm, ozaki.cuh) with s digit planes.  Only the 128 x 128 diagonal
// blocks are factored (and inverted) in native FP64, alpha comes from the
// FP64 triangular solves, the loss from the FP64 diagonal of L.  The
// result carries the digits' truncation error, about 2^-7 254^-(s-1)
// relative to each block's maximum, instead of the 2^-11 of a TF32 working
// copy, so mean and variance stay near the FP64 path with no refinement.
//
// Schedule (the same look-ahead as the TF32/BF16 path, reference
// right_looking_cholesky_tiled, core/src/cpu/tiled_algorithms.cpp:14-57):
// outer panels of 2048 columns (measured best at n = 32768 among 1024 to
// 4096, with the whole pipeline timed), inside a panel left-looking over
// 128-column blocks.  Per block column r0:
//   update   K[r0:n, r0:r0+128] -= L[r0:n, K0:r0] L[r0:r0+128, K0:r0]^T
//   potrf    L_kk and Linv_k in FP64 (potrf_diag)
//   split    Linv_k -> block digits; the panel block below -> row digits
//   solve    L[r0+128:n, r0:r0+128] = P Linv_k^T
//   split    the solved block column -> row digits (A role) and block digits (B role)
// The side stream (high priority) factors panel k+1 while the main stream
// runs the trailing update of everything right of it with panel k.
#include "gp_state.cuh"

#include <algorithm>
#include <cstdlib>
#include <string>

namespace gprat_cu
{
namespace
{

#ifndef GPRAT_OZ_PANEL_BLOCKS
#define GPRAT_OZ_PANEL_BLOCKS 16  // outer panels of 16 x 128 columns
#endif
#ifndef GPRAT_OZ_MAIN_PERCENT
#define GPRAT_OZ_MAIN_PERCENT 80  // SMs the trailing update holds while the side stream works
#endif

// Digit-plane operands of one handle (TMA maps built per call: cheap host work).
struct OzOps
{
    OzOperand LR;   // rows of L, row exponents (A role), n x n
    OzOperand LB;   // rows of L, block exponents (B role), n x n
    OzOperand INV;  // diagonal-block inverses, block exponents (B role), nblk*128 x 128
    OzOperand P;    // one unsolved panel block, row exponents (A role), n x 128
};

OzOps make_oz_ops(gprat_cu_gp *gp)
{
    const int n = gp->n, S = gp->oz_slices;
    const int64_t nn = static_cast<int64_t>(n) * n;
    const int nkb = n / OZ_KB;
    gp->oz_lr.ensure(S * nn);
    gp->oz_lb.ensure(S * nn);
    gp->oz_lr_e.ensure(static_cast<int64_t>(n) * nkb);
    gp->oz_lb_e.ensure(static_cast<int64_t>(nkb) * nkb);
    gp->oz_inv.ensure(static_cast<int64_t>(S) * gp->nblk * NB * NB);
    gp->oz_inv_e.ensure(gp->nblk);
    gp->oz_p.ensure(static_cast<int64_t>(S) * n * OZ_KB);
    gp->oz_p_e.ensure(n);
    OzOps o;
    oz_make_operand(o.LR, gp->oz_lr.ptr, gp->oz_lr_e.ptr, n, n, n, nn, nkb, S, false);
    oz_make_operand(o.LB, gp->oz_lb.ptr, gp->oz_lb_e.ptr, n, n, n, nn, nkb, S, true);
    oz_make_operand(o.INV, gp->oz_inv.ptr, gp->oz_inv_e.ptr, gp->nblk * NB, NB, NB,
                    static_cast<int64_t>(gp->nblk) * NB * NB, 1, S, true);
    oz_make_operand(o.P, gp->oz_p.ptr, gp->oz_p_e.ptr, n, OZ_KB, OZ_KB, static_cast<int64_t>(n) * OZ_KB, 1, S, false);
    return o;
}

OzGemmArgs oz_args(int M, int N, int K, int ar, int ac, int br, int bc, double *C, int64_t ldc, double alpha,
                   double beta, bool lower, DeviceStatus *st, int max_ctas = 0, double *rowsq = nullptr,
                   int64_t rowsq_half = 0)
{
    OzGemmArgs g{};
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
    g.status = st;
    g.max_ctas = max_ctas;
    g.rowsq = rowsq;
    g.rowsq_half = rowsq_half;
    return g;
}

double *kat(gprat_cu_gp *gp, int r, int c) { return gp->K.ptr + static_cast<int64_t>(r) * gp->ld + c; }

}  // namespace

void solve_alpha_fp64(gprat_cu_gp *gp, cudaStream_t s, int max_ctas)
{
    GPRAT_CUDA_CHECK(
        cudaMemcpyAsync(gp->alpha.ptr, gp->y.ptr, gp->n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    gp->flags.ensure(2);
    gp->trsv_b.ensure(gp->n);
    {
        StepScope step("forward", s);
        trsv_fused_forward(gp->K.ptr, gp->ld, gp->Linv.ptr, gp->n, gp->alpha.ptr, gp->flags.ptr, gp->trsv_b.ptr,
                           gp->status.ptr, s, max_ctas);
    }
    StepScope step("backward", s);
    trsv_fused_backward(gp->K.ptr, gp->ld, gp->Linv.ptr, gp->n, gp->alpha.ptr, gp->flags.ptr, gp->trsv_b.ptr,
                        gp->status.ptr, s, max_ctas);
}

void factor_oz(gprat_cu_gp *gp, cudaStream_t s, const std::vector<std::pair<int, cudaEvent_t>> &splits)
{
    const int n = gp->n;
    if (n % NB != 0)
    {
        throw Error(GPRAT_CU_ERR_INVALID_ARG,
                    "the int8-emulated FP64 mode needs n_tiles * n_tile_size to be a multiple of 128 (got " +
                        std::to_string(n) + ")");
    }
    const int64_t ld = gp->ld;
    const OzOps ops = make_oz_ops(gp);
    const int nbo = NB * knob("GPRAT_CU_OZ_PANEL_BLOCKS", GPRAT_OZ_PANEL_BLOCKS, 1, 64);
    const int nout = ceil_div(n, nbo);
    ensure_lookahead(gp, lookahead_events(n));
    cudaStream_t side = gp->side;
    auto evF = [&](int k) { return gp->events[1 + k]; };
    auto evR = [&](int k) { return gp->events[1 + nout + k]; };
    const int sms = device_sm_count();
    const int main_ctas = std::max(2, sms * sm_percent("GPRAT_CU_OZ_MAIN_PERCENT", GPRAT_OZ_MAIN_PERCENT) / 100);
    // digit groups of the trailing updates (0 = every group); the panel chain
    // (in-panel updates, panel solves) always keeps every group: the factor's
    // accuracy near the diagonal sets alpha's
    const int fg = std::min(gp->oz_slices, gp->oz_factor_groups);
    DeviceStatus *st = gp->status.ptr;

    {
        StepScope step("assembly", s);
        assemble_covariance(gp->x.ptr, n, gp->d, gp->T, gp->params.ptr, gp->K.ptr, ld, s);
    }
    StepScope step("cholesky", s);
    GPRAT_CUDA_CHECK(cudaEventRecord(gp->events[0], s));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(side, gp->events[0], 0));

    // factor the block columns of panel [K0, pend) on the side stream
    auto factor_panel = [&](int K0, int pend)
    {
        for (int r0 = K0; r0 < pend; r0 += NB)
        {
            const int k = r0 / NB;
            if (r0 > K0)
            {
                oz_gemm(ops.LR, ops.LB, oz_args(n - r0, NB, r0 - K0, r0, K0, r0, K0, kat(gp, r0, r0), ld, -1.0, 1.0,
                                                false, st),
                        side);
            }
            double *linv = gp->Linv.ptr + static_cast<int64_t>(k) * NB * NB;
            potrf_diag(kat(gp, r0, r0), ld, NB, r0, linv, NB, st, side);
            // every block's inverse, the last one included: the variance solve's last leaf uses it
            oz_split(linv, NB, NB, NB, nullptr, &ops.INV, k * NB, 0, side);
            const int rows = n - r0 - NB;
            if (rows <= 0)
            {
                continue;
            }
            oz_split(kat(gp, r0 + NB, r0), ld, rows, NB, &ops.P, nullptr, 0, 0, side);
            oz_gemm(ops.P, ops.INV,
                    oz_args(rows, NB, NB, 0, 0, k * NB, 0, kat(gp, r0 + NB, r0), ld, 1.0, 0.0, false, st), side);
            oz_split(kat(gp, r0 + NB, r0), ld, rows, NB, &ops.LR, &ops.LB, r0 + NB, r0, side);
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
    factor_panel(0, std::min(nbo, n));
    maybe_split(std::min(nbo, n));
    GPRAT_CUDA_CHECK(cudaEventRecord(evF(0), side));
    for (int k = 0; k < nout; ++k)
    {
        const int K0 = k * nbo;
        const int pend = std::min(K0 + nbo, n);
        const int bo = pend - K0;
        const int next_end = std::min(pend + nbo, n);
        const int rest = n - next_end;
        const bool ahead = k + 1 < nout;
        // main: everything right of panel k+1, with panel k
        GPRAT_CUDA_CHECK(cudaStreamWaitEvent(s, evF(k), 0));
        if (rest > 0)
        {
            OzGemmArgs a = oz_args(rest, rest, bo, next_end, K0, next_end, K0, kat(gp, next_end, next_end), ld, -1.0,
                                   1.0, true, st, ahead ? main_ctas : 0);
            a.groups = fg;
            oz_gemm(ops.LR, ops.LB, a, s);
        }
        GPRAT_CUDA_CHECK(cudaEventRecord(evR(k), s));
        if (!ahead)
        {
            break;
        }
        // side: panel k applied to panel k+1's columns, then panel k+1 factored
        if (k >= 1)
        {
            GPRAT_CUDA_CHECK(cudaStreamWaitEvent(side, evR(k - 1), 0));
        }
        {
            OzGemmArgs a = oz_args(n - pend, next_end - pend, bo, pend, K0, pend, K0, kat(gp, pend, pend), ld, -1.0,
                                   1.0, false, st);
            a.groups = fg;
            oz_gemm(ops.LR, ops.LB, a, side);
        }
        factor_panel(pend, next_end);
        maybe_split(next_end);
        GPRAT_CUDA_CHECK(cudaEventRecord(evF(k + 1), side));
    }
}

namespace
{

// Below this many test rows the variance solve runs in 512-column panels
// (short GEMMs over many CTAs), at or above it by recursive halving.
constexpr int OZ_RECURSIVE_MIN_ROWS = 2048;

// One variance solve W L^T = K* in place in W (FP64, m x ld), with the row
// sums of W^2 accumulated in vacc (two column halves).
struct OzVariance
{
    gprat_cu_gp *gp;
    OzOps ops;
    OzOperand WS;  // solved columns of W, row exponents (A role), m x n
    OzOperand WP;  // one unsolved 128-column block of W, row exponents, m x 128
    double *W;
    int64_t ld;
    int m;
    int max_ctas;
    cudaStream_t s;

    // W[:, c0:c0+128) := W[:, c0:c0+128) Linv_k^T, row sums of squares into vacc,
    // then the solved block's digits
    void leaf(int c0) const
    {
        const int k = c0 / NB;
        oz_split(W + c0, ld, m, NB, &WP, nullptr, 0, 0, s);
        oz_gemm(WP, ops.INV,
                oz_args(m, NB, NB, 0, 0, k * NB, 0, W + c0, ld, 1.0, 0.0, false, gp->status.ptr, max_ctas,
                        gp->vacc.ptr, m),
                s);
        oz_split(W + c0, ld, m, NB, &WS, nullptr, 0, c0, s);
    }

    // W[:, c0:c1) -= W[:, k0:k1) L[c0:c1, k0:k1)^T
    void update(int k0, int k1, int c0, int c1) const
    {
        if (k1 <= k0 || c1 <= c0)
        {
            return;
        }
        OzGemmArgs a = oz_args(m, c1 - c0, k1 - k0, 0, k0, c0, k0, W + c0, ld, -1.0, 1.0, false, gp->status.ptr,
                               max_ctas);
        a.groups = std::min(gp->oz_slices, gp->oz_variance_groups);
        oz_gemm(WS, ops.LB, a, s);
    }

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

    void solve(int c0, int c1) const
    {
        if (c1 <= c0)
        {
            return;
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

OzVariance make_variance(gprat_cu_gp *gp, int m, int max_ctas, cudaStream_t s)
{
    const int n = gp->n, S = gp->oz_slices;
    const int mm = std::max(m, 1);
    gp->oz_w.ensure(static_cast<int64_t>(S) * mm * n);
    gp->oz_w_e.ensure(static_cast<int64_t>(mm) * (n / OZ_KB));
    gp->oz_wp.ensure(static_cast<int64_t>(S) * mm * OZ_KB);
    gp->oz_wp_e.ensure(mm);
    OzVariance v{ gp, make_oz_ops(gp), {}, {}, gp->W.ptr, gp->ld, m, max_ctas, s };
    oz_make_operand(v.WS, gp->oz_w.ptr, gp->oz_w_e.ptr, mm, n, n, static_cast<int64_t>(mm) * n, n / OZ_KB, S, false);
    oz_make_operand(v.WP, gp->oz_wp.ptr, gp->oz_wp_e.ptr, mm, OZ_KB, OZ_KB, static_cast<int64_t>(mm) * OZ_KB, 1, S,
                    false);
    return v;
}

}  // namespace

void variance_oz(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s,
                 const int64_t *row_offsets, int max_ctas, bool recursive)
{
    const int n = gp->n;
    const int parts = ceil_div(n, 128);
    gp->mean_part.ensure(static_cast<int64_t>(std::max(m, 1)) * parts);
    gp->W.ensure(static_cast<int64_t>(std::max(m, 1)) * gp->ld);
    gp->vacc.ensure(2 * static_cast<int64_t>(std::max(m, 1)));
    if (m <= 0)
    {
        return;
    }
    {
        StepScope step("prediction", s);
        assemble_cross(d_xt, m, gp->x.ptr, n, gp->d, gp->params.ptr, gp->W.ptr, gp->ld,
                       d_mean != nullptr ? gp->alpha.ptr : nullptr, d_mean != nullptr ? gp->mean_part.ptr : nullptr,
                       parts, s, row_offsets);
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
    const OzVariance v = make_variance(gp, m, max_ctas, s);
    if (recursive && m >= OZ_RECURSIVE_MIN_ROWS)
    {
        v.solve(0, n);
    }
    else
    {
        v.solve_panels(n);
    }
    finalize_variance(gp->vacc.ptr, m, gp->params.ptr, d_var, s, gp->vacc.ptr + m);
}

// Fit, mean and variance (predict_with_uncertainty) on three streams:
//   caller's stream + high-priority side stream: the factorisation;
//   low-priority variance stream: K* in FP64 from the start (copied aside
//     for the mean), then segment by segment of the factor's columns (split
//     points below) the recursive variance solve of the segment and its
//     update of every column right of it, each as soon as the factorisation
//     has finished the segment's columns, on GPRAT_CU_OZ_VARIANCE_EARLY_PERCENT
//     % of the SMs (default 100), the last segment after the factorisation;
//   side stream after the factorisation: alpha (FP64 solves) and the mean.
void fit_predict_oz(gprat_cu_gp *gp, const double *d_xt, int m, double *d_mean, double *d_var, cudaStream_t s)
{
    const int n = gp->n;
    const int ne = lookahead_events(n);
    ensure_lookahead(gp, ne);
    cudaEvent_t kx_ready = gp->events[ne - 7];
    cudaEvent_t begin = gp->events[ne - 6];
    cudaEvent_t factored = gp->events[ne - 3], refined = gp->events[ne - 2], solved = gp->events[ne - 1];
    cudaStream_t side = gp->side, vs = gp->vstream;
    const int sms = device_sm_count();
    const bool early = m >= OZ_RECURSIVE_MIN_ROWS;
    // The variance solve starts on the factor's columns [0, b_1) as soon as the
    // factorisation has finished them, then [b_1, b_2) and so on; the last
    // segment follows the factorisation.  Boundaries as fractions of n
    // (GPRAT_CU_OZ_VARIANCE_SPLITS, comma-separated, at most 8; default
    // 0.5,0.75,0.875, within 1 % of the best of the sets measured at
    // n = 32768), each rounded down to a multiple of 128.
    std::vector<int> bounds;
    {
        const char *env = std::getenv("GPRAT_CU_OZ_VARIANCE_SPLITS");
        std::string spec = env != nullptr ? env : "0.5,0.75,0.875";
        size_t pos = 0;
        while (pos <= spec.size() && bounds.size() < 8)
        {
            const size_t comma = spec.find(',', pos);
            const std::string item = spec.substr(pos, comma == std::string::npos ? std::string::npos : comma - pos);
            char *end = nullptr;
            const double f = std::strtod(item.c_str(), &end);
            if (end != item.c_str() && f > 0.0 && f < 1.0)
            {
                const int b = static_cast<int>(f * n / NB) * NB;
                if (b > (bounds.empty() ? 0 : bounds.back()) && b < n)
                {
                    bounds.push_back(b);
                }
            }
            if (comma == std::string::npos)
            {
                break;
            }
            pos = comma + 1;
        }
    }
    // buffers first (an allocation must not fall between launches of different streams)
    const int mm = std::max(m, 1);
    gp->W.ensure(static_cast<int64_t>(mm) * gp->ld);
    gp->Kx.ensure(static_cast<int64_t>(mm) * gp->ld);
    gp->vacc.ensure(2 * static_cast<int64_t>(mm));
    gp->mean_part.ensure(static_cast<int64_t>(mm) * ceil_div(n, 128));
    make_oz_ops(gp);
    const OzVariance v = make_variance(gp, m, 0, vs);
    GPRAT_CUDA_CHECK(cudaEventRecord(begin, s));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(vs, begin, 0));
    std::vector<std::pair<int, cudaEvent_t>> splits;
    if (early)
    {
        for (size_t i = 0; i < bounds.size(); ++i)
        {
            splits.emplace_back(bounds[i], gp->events[ne - 8 - static_cast<int>(i)]);
        }
    }
    factor_oz(gp, s, splits);
    GPRAT_CUDA_CHECK(cudaEventRecord(factored, s));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(side, factored, 0));
    if (m > 0)
    {
        {
            StepScope step("prediction", vs);
            assemble_cross(d_xt, m, gp->x.ptr, n, gp->d, gp->params.ptr, gp->W.ptr, gp->ld, nullptr, nullptr, 0, vs);
            GPRAT_CUDA_CHECK(cudaMemcpyAsync(gp->Kx.ptr, gp->W.ptr, static_cast<size_t>(m) * gp->ld * sizeof(double),
                                             cudaMemcpyDeviceToDevice, vs));
            GPRAT_CUDA_CHECK(cudaEventRecord(kx_ready, vs));
        }
        StepScope step("forward KcK", vs);
        GPRAT_CUDA_CHECK(cudaMemsetAsync(gp->vacc.ptr, 0, 2 * m * sizeof(double), vs));
        OzVariance w = v;
        if (early)
        {
            w.max_ctas = std::max(2, sms * sm_percent("GPRAT_CU_OZ_VARIANCE_EARLY_PERCENT", 100) / 100);
            int c0 = 0;
            for (const auto &sp : splits)
            {
                GPRAT_CUDA_CHECK(cudaStreamWaitEvent(vs, sp.second, 0));
                w.solve(c0, sp.first);
                w.update(c0, sp.first, sp.first, n);
                c0 = sp.first;
            }
            GPRAT_CUDA_CHECK(cudaStreamWaitEvent(vs, factored, 0));
            w.max_ctas = 0;
            w.solve(c0, n);
        }
        else
        {
            GPRAT_CUDA_CHECK(cudaStreamWaitEvent(vs, factored, 0));
            w.solve_panels(n);
        }
        finalize_variance(gp->vacc.ptr, m, gp->params.ptr, d_var, vs, gp->vacc.ptr + m);
    }
    GPRAT_CUDA_CHECK(cudaEventRecord(solved, vs));
    {
        StepScope step("alpha", side);
        solve_alpha_fp64(gp, side);
    }
    if (m > 0)
    {
        StepScope step("prediction", side);
        GPRAT_CUDA_CHECK(cudaStreamWaitEvent(side, kx_ready, 0));
        cross_times_alpha(gp->Kx.ptr, gp->ld, m, n, gp->alpha.ptr, d_mean, side);
    }
    GPRAT_CUDA_CHECK(cudaEventRecord(refined, side));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(s, refined, 0));
    GPRAT_CUDA_CHECK(cudaStreamWaitEvent(s, solved, 0));
}

}  // namespace gprat_cu
