// Blocked triangular solves for alpha = K^-1 y, the loss, and small helpers.
//
// forward_solve_tiled / backward_solve_tiled (core/src/cpu/tiled_algorithms.cpp:61-115)
// run a trsv per diagonal tile and a gemv per off-diagonal tile.  Here the
// diagonal-block inverses from potrf_diag make the per-block solve a small
// matrix-vector product (warp-shuffle dot products), and the off-diagonal
// updates are coalesced row (forward) or column (backward) sweeps over L,
// so each solve streams L from HBM once (memory bound).
#include "common.cuh"

namespace gprat_cu
{
namespace
{

constexpr int DT = 1024;  // threads of the diagonal-block kernels

// z = Linv * r  (rows of Linv read by whole warps; shuffle reduction)
__global__ void __launch_bounds__(DT) diag_fwd_kernel(const double *__restrict__ Linv, int nb, int bs,
                                                      double *__restrict__ r)
{
    __shared__ double rk[128];
    __shared__ double z[128];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < bs)
    {
        rk[threadIdx.x] = r[threadIdx.x];
    }
    __syncthreads();
    for (int row = warp; row < bs; row += DT / 32)
    {
        double s = 0.0;
        for (int c = lane; c <= row; c += 32)
        {
            s += Linv[row * nb + c] * rk[c];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            s += __shfl_xor_sync(0xffffffffu, s, o);
        }
        if (lane == 0)
        {
            z[row] = s;
        }
    }
    __syncthreads();
    if (threadIdx.x < bs)
    {
        r[threadIdx.x] = z[threadIdx.x];
    }
}

// a = Linv^T * r  (thread c walks column c: row reads are coalesced)
__global__ void __launch_bounds__(128) diag_bwd_kernel(const double *__restrict__ Linv, int nb, int bs,
                                                       double *__restrict__ r)
{
    __shared__ double rk[128];
    const int c = threadIdx.x;
    if (c < bs)
    {
        rk[c] = r[c];
    }
    __syncthreads();
    if (c < bs)
    {
        double s = 0.0;
        for (int p = c; p < bs; ++p)
        {
            s += Linv[p * nb + c] * rk[p];
        }
        r[c] = s;
    }
}

// r[i] -= L[i][0:bs] . z for rows i in [0, rows) (L points at the block
// column, rows start right below the diagonal block).  One warp per row.
// L may be FP64 or FP32 (the mixed-precision factor); arithmetic is FP64.
template <typename T>
__global__ void __launch_bounds__(256) fwd_update_kernel(const T *__restrict__ L, int64_t ldl, int rows, int bs,
                                                         const double *__restrict__ z, double *__restrict__ r)
{
    __shared__ double zs[128];
    if (threadIdx.x < bs)
    {
        zs[threadIdx.x] = z[threadIdx.x];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (row >= rows)
    {
        return;
    }
    const T *lr = L + static_cast<int64_t>(row) * ldl;
    double s = 0.0;
    for (int c = lane; c < bs; c += 32)
    {
        s += static_cast<double>(lr[c]) * zs[c];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if (lane == 0)
    {
        r[row] -= s;
    }
}

// r[c] -= sum_p L[p][c] * a[p] for c in [0, cols) (L points at the first
// row of the block row; rows p < bs).  Threads own columns.
template <typename T>
__global__ void __launch_bounds__(256) bwd_update_kernel(const T *__restrict__ L, int64_t ldl, int cols, int bs,
                                                         const double *__restrict__ a, double *__restrict__ r)
{
    __shared__ double as[128];
    if (threadIdx.x < bs)
    {
        as[threadIdx.x] = a[threadIdx.x];
    }
    __syncthreads();
    const int c = blockIdx.x * 256 + threadIdx.x;
    if (c >= cols)
    {
        return;
    }
    double s = 0.0;
    for (int p = 0; p < bs; ++p)
    {
        s += static_cast<double>(L[static_cast<int64_t>(p) * ldl + c]) * as[p];
    }
    r[c] -= s;
}

__global__ void __launch_bounds__(1024) loss_kernel_impl(const double *__restrict__ y, const double *__restrict__ alpha,
                                                         const double *__restrict__ L, int64_t ldl, int n,
                                                         DeviceParams *__restrict__ p)
{
    __shared__ double s1[1024];
    __shared__ double s2[1024];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < n; i += 1024)
    {
        a += y[i] * alpha[i];
        double d = L[static_cast<int64_t>(i) * ldl + i];
        b += log(d * d);
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1)
    {
        if (threadIdx.x < w)
        {
            s1[threadIdx.x] += s1[threadIdx.x + w];
            s2[threadIdx.x] += s2[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        // add_losses (core/src/cpu/gp_optimizer.cpp:205-218)
        const double two_pi = 6.283185307179586;
        double nn = static_cast<double>(n);
        double l = s1[0] + s2[0];
        l += nn * log(two_pi);
        p->loss = 0.5 * l / nn;
    }
}

__global__ void finalize_var_kernel(const double *__restrict__ acc, const double *__restrict__ acc2, int m,
                                    const DeviceParams *__restrict__ p, double *__restrict__ var)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < m)
    {
        // gen_tile_prior_covariance gives k(x,x) = v (core/src/cpu/gp_algorithms.cpp:90-111)
        const double a = acc2 != nullptr ? acc[r] + acc2[r] : acc[r];
        var[r] = p->hyper[1] - a;
    }
}

__global__ void set_params_kernel(DeviceParams *p, DeviceParams v) { *p = v; }

__global__ void diag_ones_kernel(double *A, int64_t lda, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        A[static_cast<int64_t>(i) * lda + i] = 1.0;
    }
}

}  // namespace

namespace
{

template <typename T>
void trsv_forward_t(const T *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, cudaStream_t s)
{
    const int nblk = ceil_div(n, nb);
    for (int k = 0; k < nblk; ++k)
    {
        const int r0 = k * nb;
        const int bs = min(nb, n - r0);
        diag_fwd_kernel<<<1, DT, 0, s>>>(Linv + static_cast<int64_t>(k) * nb * nb, nb, bs, rhs + r0);
        GPRAT_LAUNCH_CHECK();
        const int rows = n - r0 - bs;
        if (rows > 0)
        {
            fwd_update_kernel<<<ceil_div(rows, 8), 256, 0, s>>>(L + static_cast<int64_t>(r0 + bs) * ldl + r0, ldl, rows,
                                                                bs, rhs + r0, rhs + r0 + bs);
            GPRAT_LAUNCH_CHECK();
        }
    }
}

template <typename T>
void trsv_backward_t(const T *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, cudaStream_t s)
{
    const int nblk = ceil_div(n, nb);
    for (int k = nblk - 1; k >= 0; --k)
    {
        const int r0 = k * nb;
        const int bs = min(nb, n - r0);
        diag_bwd_kernel<<<1, 128, 0, s>>>(Linv + static_cast<int64_t>(k) * nb * nb, nb, bs, rhs + r0);
        GPRAT_LAUNCH_CHECK();
        if (r0 > 0)
        {
            bwd_update_kernel<<<ceil_div(r0, 256), 256, 0, s>>>(L + static_cast<int64_t>(r0) * ldl, ldl, r0, bs,
                                                                rhs + r0, rhs);
            GPRAT_LAUNCH_CHECK();
        }
    }
}

}  // namespace

void trsv_forward(const double *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, double *, cudaStream_t s)
{
    trsv_forward_t(L, ldl, Linv, nb, n, rhs, s);
}

void trsv_backward(const double *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, double *,
                   cudaStream_t s)
{
    trsv_backward_t(L, ldl, Linv, nb, n, rhs, s);
}

void trsv_forward_f32(const float *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, cudaStream_t s)
{
    trsv_forward_t(L, ldl, Linv, nb, n, rhs, s);
}

void trsv_backward_f32(const float *L, int64_t ldl, const double *Linv, int nb, int n, double *rhs, cudaStream_t s)
{
    trsv_backward_t(L, ldl, Linv, nb, n, rhs, s);
}

void loss_kernel(const double *y, const double *alpha, const double *L, int64_t ldl, int n, DeviceParams *p,
                 cudaStream_t s)
{
    loss_kernel_impl<<<1, 1024, 0, s>>>(y, alpha, L, ldl, n, p);
    GPRAT_LAUNCH_CHECK();
}

void finalize_variance(const double *acc, int m, const DeviceParams *p, double *var, cudaStream_t s,
                       const double *acc2)
{
    if (m <= 0)
    {
        return;
    }
    finalize_var_kernel<<<ceil_div(m, 256), 256, 0, s>>>(acc, acc2, m, p, var);
    GPRAT_LAUNCH_CHECK();
}

void set_params(DeviceParams *p, const DeviceParams &value, cudaStream_t s)
{
    set_params_kernel<<<1, 1, 0, s>>>(p, value);
    GPRAT_LAUNCH_CHECK();
}

void set_identity(double *A, int64_t lda, int n, cudaStream_t s)
{
    GPRAT_CUDA_CHECK(cudaMemset2DAsync(A, lda * sizeof(double), 0, n * sizeof(double), n, s));
    diag_ones_kernel<<<ceil_div(n, 256), 256, 0, s>>>(A, lda, n);
    GPRAT_LAUNCH_CHECK();
}

void copy_rows(const double *src, int64_t lds, double *dst, int64_t ldd, int rows, int cols, cudaStream_t s)
{
    GPRAT_CUDA_CHECK(cudaMemcpy2DAsync(dst, ldd * sizeof(double), src, lds * sizeof(double), cols * sizeof(double),
                                       rows, cudaMemcpyDeviceToDevice, s));
}

}  // namespace gprat_cu
