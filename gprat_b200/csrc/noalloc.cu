// Loss entry point that allocates no memory (gprat_cu_compute_loss_noalloc).
//
// Some callers cannot call cudaMalloc: code running while a memory pool or
// allocator it does not own is in charge of the device (for example inside
// another framework's allocator, or a real-time loop that must not hit the
// driver's allocator and its implicit synchronisation).  This entry point
// computes the same loss as gprat_cu_compute_loss on caller-provided device
// buffers, and keeps all of its scratch (covariance / Cholesky factor,
// diagonal-block inverses, alpha, parameter block, status word) in one
// file-scope device array of fixed size.  Nothing is allocated: no
// cudaMalloc, no cudaFree, no allocating library routine.
//
// Limits and sharing:
//   * n_tiles * n_tile_size must not exceed NOALLOC_MAX_N (1024); larger
//     problems are rejected with GPRAT_CU_ERR_INVALID_ARG.
//   * Every GPU that loads the library holds the array (about 9.4 MB) until
//     the process exits.
//   * All calls share the array and it keeps the last call's contents; the
//     status word is cleared at the start of every call and every other
//     region is fully rewritten before it is read.  Calls that overlap on
//     the GPU (different streams or threads, same device) race on it.
//   * The first call on a device resolves the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current).
//     Every call reads the status word back and synchronises its stream, so
//     no call can be captured into a CUDA graph.  With CUDA's lazy
//     module loading (the default) that first call may also load the
//     library's device code and so reserve the array: a caller that must
//     never allocate makes one warm-up call outside its critical region.
//     The address is kept for the life of the process, so cudaDeviceReset
//     on a device after its first call is not supported.
//   * Every call copies the status word to the host and synchronises the
//     stream it was given before it returns.
#include "common.cuh"
#include "gprat_cu.h"

#include <cstring>
#include <mutex>
#include <string>

namespace
{

using namespace gprat_cu;

constexpr int NB = 128;
constexpr int64_t NOALLOC_MAX_N = 1024;
constexpr int64_t OFF_K = 0;                                                 // n x ld doubles
constexpr int64_t OFF_LINV = OFF_K + NOALLOC_MAX_N * NOALLOC_MAX_N;          // nblk x 128 x 128
constexpr int64_t OFF_ALPHA = OFF_LINV + (NOALLOC_MAX_N / NB) * NB * NB;     // n
constexpr int64_t OFF_PARAMS = OFF_ALPHA + NOALLOC_MAX_N;                    // DeviceParams
constexpr int64_t OFF_STATUS = OFF_PARAMS + 32;                              // DeviceStatus
constexpr int64_t SCRATCH_DOUBLES = OFF_STATUS + 32;
static_assert(sizeof(DeviceParams) <= 32 * sizeof(double), "parameter block does not fit its slot");
static_assert(sizeof(DeviceStatus) <= 32 * sizeof(double), "status word does not fit its slot");

// The scratch.  In host code this name is only a host-side stand-in, not a
// device address: host code must use the address from cudaGetSymbolAddress.
static __device__ __align__(256) double g_scratch[SCRATCH_DOUBLES];

std::mutex g_addr_mtx;
double *g_addr[64] = {};

double *scratch_address(int device)
{
    if (device < 0 || device >= 64)
    {
        throw Error(GPRAT_CU_ERR_INVALID_ARG, "device index out of range for the no-allocation scratch");
    }
    std::lock_guard<std::mutex> lk(g_addr_mtx);
    if (g_addr[device] == nullptr)
    {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || p == nullptr)
        {
            throw Error(GPRAT_CU_ERR_CUDA,
                        std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") + cudaGetErrorString(e));
        }
        g_addr[device] = static_cast<double *>(p);
    }
    return g_addr[device];
}

}  // namespace

namespace gprat_cu
{
void set_last_error(const std::string &message);  // gp.cu: text for gprat_cu_last_error()
}

extern "C" int gprat_cu_compute_loss_noalloc(int device,
                                             const double *d_train_in,
                                             int64_t n_in,
                                             const double *d_train_out,
                                             int64_t n_out,
                                             int n_tiles,
                                             int n_tile_size,
                                             int n_regressors,
                                             const double hyper[3],
                                             double *d_loss,
                                             void *stream)
{
    try
    {
        if (d_train_in == nullptr || d_train_out == nullptr || d_loss == nullptr || hyper == nullptr)
        {
            throw Error(GPRAT_CU_ERR_INVALID_ARG, "inputs and output must not be NULL");
        }
        if (n_tiles <= 0 || n_tile_size <= 0 || n_regressors <= 0)
        {
            throw Error(GPRAT_CU_ERR_INVALID_ARG, "n_tiles, n_tile_size and n_regressors must be positive");
        }
        const int64_t n64 = static_cast<int64_t>(n_tiles) * n_tile_size;
        if (n64 > NOALLOC_MAX_N)
        {
            throw Error(GPRAT_CU_ERR_INVALID_ARG, "n_tiles * n_tile_size = " + std::to_string(n64) +
                                                      " exceeds the no-allocation limit of " +
                                                      std::to_string(NOALLOC_MAX_N) + " training points");
        }
        if (n_in < n64 + n_regressors - 1 || n_out < n64)
        {
            throw Error(GPRAT_CU_ERR_INVALID_ARG, "training input or output too short");
        }
        const int n = static_cast<int>(n64);
        const int64_t ld = round_up(n, 8);
        const int nblk = ceil_div(n, NB);

        int prev = -1;
        GPRAT_CUDA_CHECK(cudaGetDevice(&prev));
        if (prev != device)
        {
            GPRAT_CUDA_CHECK(cudaSetDevice(device));
        }
        struct Restore
        {
            int dev;
            ~Restore()
            {
                if (dev >= 0)
                {
                    cudaSetDevice(dev);
                }
            }
        } restore{ prev != device ? prev : -1 };

        double *base = scratch_address(device);
        double *K = base + OFF_K;
        double *Linv = base + OFF_LINV;
        double *alpha = base + OFF_ALPHA;
        auto *params = reinterpret_cast<DeviceParams *>(base + OFF_PARAMS);
        auto *status = reinterpret_cast<DeviceStatus *>(base + OFF_STATUS);
        cudaStream_t s = static_cast<cudaStream_t>(stream);

        DeviceParams v;
        std::memset(&v, 0, sizeof(v));
        for (int q = 0; q < 3; ++q)
        {
            v.hyper[q] = hyper[q];
        }
        set_params(params, v, s);
        GPRAT_CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(DeviceStatus), s));

        assemble_covariance(d_train_in, n, n_regressors, n_tile_size, params, K, ld, s);
        for (int k = 0; k < nblk; ++k)
        {
            const int r0 = k * NB;
            const int bs = std::min(NB, n - r0);
            double *Lk = Linv + static_cast<int64_t>(k) * NB * NB;
            potrf_diag(K + r0 * ld + r0, ld, bs, r0, Lk, NB, status, s);
            const int rows = n - r0 - bs;
            if (rows <= 0)
            {
                continue;
            }
            GemmArgs pa{};
            pa.M = rows;
            pa.N = bs;
            pa.K = bs;
            pa.A = K + (r0 + bs) * ld + r0;
            pa.lda = ld;
            pa.B = Lk;
            pa.ldb = NB;
            pa.transB = true;
            pa.C = K + (r0 + bs) * ld + r0;
            pa.ldc = ld;
            pa.alpha = 1.0;
            pa.beta = 0.0;
            dgemm(pa, s);
            GemmArgs ta{};
            ta.M = rows;
            ta.N = rows;
            ta.K = bs;
            ta.A = K + (r0 + bs) * ld + r0;
            ta.lda = ld;
            ta.B = K + (r0 + bs) * ld + r0;
            ta.ldb = ld;
            ta.transB = true;
            ta.C = K + (r0 + bs) * ld + r0 + bs;
            ta.ldc = ld;
            ta.alpha = -1.0;
            ta.beta = 1.0;
            ta.lower = true;
            dgemm(ta, s);
        }
        GPRAT_CUDA_CHECK(cudaMemcpyAsync(alpha, d_train_out, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        trsv_forward(K, ld, Linv, NB, n, alpha, nullptr, s);
        trsv_backward(K, ld, Linv, NB, n, alpha, nullptr, s);
        loss_kernel(d_train_out, alpha, K, ld, n, params, s);
        GPRAT_CUDA_CHECK(cudaMemcpyAsync(d_loss, &params->loss, sizeof(double), cudaMemcpyDeviceToDevice, s));
        DeviceStatus st{};
        GPRAT_CUDA_CHECK(cudaMemcpyAsync(&st, status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, s));
        GPRAT_CUDA_CHECK(cudaStreamSynchronize(s));
        if (st.not_spd_row != 0)
        {
            throw Error(GPRAT_CU_ERR_NOT_SPD, "Cholesky factorisation failed: covariance matrix is not positive "
                                              "definite (non-positive pivot at row " +
                                                  std::to_string(st.not_spd_row - 1) + ")");
        }
        set_last_error("");
        return GPRAT_CU_OK;
    }
    catch (const Error &e)
    {
        set_last_error(e.what());
        return e.code;
    }
    catch (const std::exception &e)
    {
        set_last_error(e.what());
        return GPRAT_CU_ERR_INVALID_ARG;
    }
}
