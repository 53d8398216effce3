// Kernel-level test entry points of the C ABI (gprat_cu_test_*): run one
// kernel on host-provided data so that tests can compare it in isolation.
#include "gprat_cu.h"
#include "tc_gemm.cuh"

#include <string>
#include <vector>

namespace gprat_cu
{
void set_last_error(const std::string &message);
}

namespace
{

using namespace gprat_cu;

struct Buf
{
    void *p = nullptr;
    explicit Buf(size_t bytes)
    {
        GPRAT_CUDA_CHECK(cudaMalloc(&p, bytes));
    }
    ~Buf()
    {
        if (p != nullptr)
        {
            cudaFree(p);
        }
    }
    Buf(const Buf &) = delete;
    Buf &operator=(const Buf &) = delete;
};

}  // namespace

extern "C" int gprat_cu_test_tc_gemm(int kind, int M, int N, int K, const float *A, int64_t lda, const float *B,
                                     int64_t ldb, float *C, int64_t ldc, float alpha, float beta, int lower,
                                     double *rowsq, int tile_mode)
{
    try
    {
        if (A == nullptr || B == nullptr || C == nullptr || M <= 0 || N <= 0 || K <= 0 || lda < K || ldb < K ||
            ldc < N || (kind != 0 && kind != 1) || tile_mode < 0 || tile_mode > 3)
        {
            throw Error(GPRAT_CU_ERR_INVALID_ARG, "gprat_cu_test_tc_gemm: invalid arguments");
        }
        cudaStream_t s = nullptr;
        // device copies with padded leading dimensions (multiples of 64 elements)
        const int64_t la = round_up(K, 64), lb = round_up(K, 64), lc = round_up(N, 4);
        Buf dA(static_cast<size_t>(M) * la * 4), dB(static_cast<size_t>(N) * lb * 4), dC(static_cast<size_t>(M) * lc * 4);
        GPRAT_CUDA_CHECK(cudaMemcpy2D(dA.p, la * 4, A, lda * 4, K * 4, M, cudaMemcpyHostToDevice));
        GPRAT_CUDA_CHECK(cudaMemcpy2D(dB.p, lb * 4, B, ldb * 4, K * 4, N, cudaMemcpyHostToDevice));
        GPRAT_CUDA_CHECK(cudaMemcpy2D(dC.p, lc * 4, C, ldc * 4, N * 4, M, cudaMemcpyHostToDevice));
        Buf dStatus(sizeof(DeviceStatus));
        GPRAT_CUDA_CHECK(cudaMemset(dStatus.p, 0, sizeof(DeviceStatus)));
        // two column-half accumulators: the caller's values in the first, zeros in the second
        Buf dRow(2 * static_cast<size_t>(M) * sizeof(double));
        if (rowsq != nullptr)
        {
            GPRAT_CUDA_CHECK(cudaMemset(dRow.p, 0, 2 * static_cast<size_t>(M) * sizeof(double)));
            GPRAT_CUDA_CHECK(cudaMemcpy(dRow.p, rowsq, M * sizeof(double), cudaMemcpyHostToDevice));
        }
        TcOperand oa, ob;
        Buf hA(kind == 1 ? static_cast<size_t>(M) * la * 2 : 16), hB(kind == 1 ? static_cast<size_t>(N) * lb * 2 : 16);
        if (kind == 1)
        {
            convert_f32_to_bf16(static_cast<const float *>(dA.p), la, hA.p, la, M, K, s);
            convert_f32_to_bf16(static_cast<const float *>(dB.p), lb, hB.p, lb, N, K, s);
            tc_make_operand(oa, hA.p, M, static_cast<int>(la), la, TcKind::BF16);
            tc_make_operand(ob, hB.p, N, static_cast<int>(lb), lb, TcKind::BF16);
        }
        else
        {
            tc_make_operand(oa, dA.p, M, static_cast<int>(la), la, TcKind::TF32);
            tc_make_operand(ob, dB.p, N, static_cast<int>(lb), lb, TcKind::TF32);
        }
        TcGemmArgs g{};
        g.M = M;
        g.N = N;
        g.K = K;
        g.C = static_cast<float *>(dC.p);
        g.ldc = lc;
        g.alpha = alpha;
        g.beta = beta;
        g.lower = lower != 0;
        g.rowsq = rowsq != nullptr ? static_cast<double *>(dRow.p) : nullptr;
        g.rowsq_half = M;
        g.tile_mode = tile_mode;
        g.status = static_cast<DeviceStatus *>(dStatus.p);
        tc_gemm(oa, ob, g, s);
        GPRAT_CUDA_CHECK(cudaStreamSynchronize(s));
        DeviceStatus st{};
        GPRAT_CUDA_CHECK(cudaMemcpy(&st, dStatus.p, sizeof(st), cudaMemcpyDeviceToHost));
        if (st.timeout != 0)
        {
            throw Error(GPRAT_CU_ERR_TIMEOUT, "tensor-core GEMM: a bounded wait timed out");
        }
        GPRAT_CUDA_CHECK(cudaMemcpy2D(C, ldc * 4, dC.p, lc * 4, N * 4, M, cudaMemcpyDeviceToHost));
        if (rowsq != nullptr)
        {
            std::vector<double> halves(2 * static_cast<size_t>(M));
            GPRAT_CUDA_CHECK(cudaMemcpy(halves.data(), dRow.p, halves.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (int i = 0; i < M; ++i)
            {
                rowsq[i] = halves[i] + halves[M + i];
            }
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
