// Adjoint gradient of the NLML and the Adam step, on the device.
//
// Reference (core/src/cpu/gp_functions.cpp:1032-1269, tiled_algorithms.cpp:296-448):
// materialise dK/dl and dK/dv tiles (gp_optimizer.cpp:115-150), form the
// explicit K^-1 by two tiled solves on the identity (2n^3 flops), then
//   g_theta = s_theta * 0.5/N * (tr(K^-1 dK) - alpha^T dK alpha),
//   g_noise = s_noise * 0.5/N * (tr(K^-1) - alpha^T alpha),
// with s = sigmoid(softplus^-1(theta)), and apply Adam on the unconstrained
// parameters (gp_optimizer.cpp:154-183).
//
// Here K^-1 = U U^T with U = L^-T (computed by the blocked solve W L^T = I,
// n^3/3 flops).  One fused kernel then forms each lower tile of U U^T on
// the DMMA tensor cores and, in its epilogue, regenerates the distance
// d_ij = -r_ij^2/(2 l^2) from the series, e_ij = exp(d_ij), and reduces
//   sum w_ij (K^-1_ij - a_i a_j) * (-2 v/l) d_ij e_ij,
//   sum w_ij (K^-1_ij - a_i a_j) * e_ij,       sum_i (K^-1_ii - a_i^2)
// (w = 2 off the diagonal, 1 on it).  Neither K^-1 nor the derivative
// matrices are ever stored.  A single-thread kernel then reduces the
// per-tile partials in a fixed order and applies Adam to the device-resident
// parameters, so an optimisation loop never returns to the host.
#include "dgemm.cuh"

namespace gprat_cu
{
namespace
{

using namespace gemm;
using AC = Cfg<4>;  // 128x128 tiles, 8 warps
constexpr int THREADS = AC::THREADS;
constexpr int BM = AC::BM;
constexpr int BN = AC::BN;

__global__ void __launch_bounds__(THREADS, 1) adjoint_kernel(GemmArgs a, const double *__restrict__ alpha,
                                                             const double *__restrict__ x, int d,
                                                             const DeviceParams *__restrict__ p,
                                                             double *__restrict__ partials)
{
    extern __shared__ __align__(16) double smem[];
    TileCoord tc = tile_coord<BM, BN>(true);
    const int m0 = tc.m0, n0 = tc.n0;
    Frag f = frag_coords<4>();
    double acc[4][4][4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                acc[mi][ni][q] = 0.0;

    // U is upper triangular: rows >= m0 vanish for p < m0.
    mainloop<4, false, true>(a, m0, n0, smem, acc, (m0 / BK) * BK, f);

    // stage series windows and alpha for the tile's rows and columns
    double *xr = smem;
    double *xc = xr + BM + d;
    double *ar = xc + BN + d;
    double *ac = ar + BM;
    double *red = ac + BN;  // 3 x THREADS/32
    const int n = a.M;
    for (int q = threadIdx.x; q < BM + d - 1; q += THREADS)
    {
        int g = m0 + q;
        xr[q] = (g < n + d - 1) ? x[g] : 0.0;
    }
    for (int q = threadIdx.x; q < BN + d - 1; q += THREADS)
    {
        int g = n0 + q;
        xc[q] = (g < n + d - 1) ? x[g] : 0.0;
    }
    for (int q = threadIdx.x; q < BM; q += THREADS)
    {
        ar[q] = (m0 + q < n) ? alpha[m0 + q] : 0.0;
        ac[q] = (n0 + q < n) ? alpha[n0 + q] : 0.0;
    }
    __syncthreads();

    const double l = p->hyper[0];
    const double v = p->hyper[1];
    const double nh = -0.5 / (l * l);
    const double fl = -2.0 * v / l;
    double gl = 0.0, gv = 0.0, gn = 0.0;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
    {
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
        {
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                int li = f.wm * 64 + mi * 16 + f.g + (q >> 1) * 8;
                int lj = f.wn * 32 + ni * 8 + 2 * f.t + (q & 1);
                int i = m0 + li, j = n0 + lj;
                if (i >= n || j >= n || j > i)
                {
                    continue;
                }
                double dist = 0.0;
                for (int k = 0; k < d; ++k)
                {
                    double z = __dsub_rn(xr[li + k], xc[lj + k]);
                    dist = __dadd_rn(dist, __dmul_rn(z, z));
                }
                double dd = __dmul_rn(nh, dist);
                double e = exp(dd);
                double w = (i == j) ? 1.0 : 2.0;
                double qv = acc[mi][ni][q] - ar[li] * ac[lj];
                gl += w * qv * (fl * dd * e);
                gv += w * qv * e;
                if (i == j)
                {
                    gn += qv;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        gl += __shfl_xor_sync(0xffffffffu, gl, o);
        gv += __shfl_xor_sync(0xffffffffu, gv, o);
        gn += __shfl_xor_sync(0xffffffffu, gn, o);
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
    {
        red[warp] = gl;
        red[THREADS / 32 + warp] = gv;
        red[2 * THREADS / 32 + warp] = gn;
    }
    __syncthreads();
    if (threadIdx.x < 3)
    {
        double s = 0.0;
        for (int w = 0; w < THREADS / 32; ++w)
        {
            s += red[threadIdx.x * (THREADS / 32) + w];
        }
        partials[blockIdx.x * 3 + threadIdx.x] = s;
    }
}

__device__ double to_constrained(double u, bool noise)
{
    // core/src/cpu/gp_optimizer.cpp:12-22
    return noise ? log(1.0 + exp(u)) + 1e-6 : log(1.0 + exp(u));
}

__device__ double to_unconstrained(double t, bool noise)
{
    // core/src/cpu/gp_optimizer.cpp:24-34
    return noise ? log(exp(t - 1e-6) - 1.0) : log(exp(t) - 1.0);
}

__device__ double sigmoid(double u) { return 1.0 / (1.0 + exp(-u)); }

__global__ void adjoint_finish_kernel(const double *__restrict__ partials, int np, int n, DeviceParams *__restrict__ p,
                                      int adam_step)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
    {
        return;
    }
    double G[3] = { 0.0, 0.0, 0.0 };
    for (int b = 0; b < np; ++b)
    {
        G[0] += partials[3 * b + 0];
        G[1] += partials[3 * b + 1];
        G[2] += partials[3 * b + 2];
    }
    const double scale = 0.5 / static_cast<double>(n);  // compute_gradient (gp_optimizer.cpp:222-225)
    double g[3];
    g[0] = sigmoid(to_unconstrained(p->hyper[0], false)) * (scale * G[0]);
    g[1] = sigmoid(to_unconstrained(p->hyper[1], false)) * (scale * G[1]);
    g[2] = sigmoid(to_unconstrained(p->hyper[2], true)) * (scale * G[2]);
    for (int q = 0; q < 3; ++q)
    {
        p->grad[q] = g[q];
    }
    if (!adam_step)
    {
        return;
    }
    const double lr = p->adam[0], b1 = p->adam[1], b2 = p->adam[2], eps = p->adam[3];
    for (int q = 0; q < 3; ++q)
    {
        if (!p->trainable[q])
        {
            continue;
        }
        // update_first/second_moment, adam_step (gp_optimizer.cpp:154-183)
        p->m_T[q] = b1 * p->m_T[q] + (1.0 - b1) * g[q];
        p->w_T[q] = b2 * p->w_T[q] + (1.0 - b2) * g[q] * g[q];
        const bool jitter = (q == 2);
        double u = to_unconstrained(p->hyper[q], jitter);
        double b1t = pow(b1, static_cast<double>(p->iter + 1));
        double b2t = pow(b2, static_cast<double>(p->iter + 1));
        double nu = lr * sqrt(1.0 - b2t) / (1.0 - b1t);
        u = u - nu * p->m_T[q] / (sqrt(p->w_T[q]) + eps);
        p->hyper[q] = to_constrained(u, jitter);
    }
    p->iter += 1;
}

}  // namespace

void adjoint_trace(const double *U, int64_t ldu, const double *alpha, const double *x, int n, int n_reg,
                   const DeviceParams *p, double *partials, int *n_partials, cudaStream_t s)
{
    GemmArgs a{};
    a.M = n;
    a.N = n;
    a.K = n;
    a.A = U;
    a.lda = ldu;
    a.transA = false;
    a.B = U;
    a.ldb = ldu;
    a.transB = true;
    a.C = nullptr;
    a.ldc = 0;
    a.alpha = 1.0;
    a.beta = 0.0;
    a.lower = true;
    a.rowsq = nullptr;
    a.k_tri = 1;
    if ((ldu & 1) || (reinterpret_cast<uintptr_t>(U) & 15))
    {
        throw Error(1, "adjoint_trace: U must be 16-byte aligned with an even leading dimension");
    }
    constexpr int smem_main = smem_bytes<4, false, true>();
    const int smem_epi = static_cast<int>((BM + BN + 2 * n_reg + BM + BN + 3 * THREADS / 32) * sizeof(double));
    const int smem = smem_main > smem_epi ? smem_main : smem_epi;
    if (smem > 227 * 1024)
    {
        throw Error(1, "adjoint_trace: too many regressors");
    }
    ensure_smem_attr(reinterpret_cast<const void *>(adjoint_kernel), smem);
    const int t = ceil_div(n, BM);
    const int tiles = t * (t + 1) / 2;
    adjoint_kernel<<<tiles, THREADS, smem, s>>>(a, alpha, x, n_reg, p, partials);
    GPRAT_LAUNCH_CHECK();
    *n_partials = tiles;
}

void adjoint_finish(const double *partials, int n_partials, int n, DeviceParams *p, bool adam_step, cudaStream_t s)
{
    adjoint_finish_kernel<<<1, 32, 0, s>>>(partials, n_partials, n, p, adam_step ? 1 : 0);
    GPRAT_LAUNCH_CHECK();
}

}  // namespace gprat_cu
