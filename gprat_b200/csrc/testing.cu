// Kernel-level test entry points of the C ABI (gprat_cu_test_*): run one
// kernel on host-provided data so that tests can compare it in isolation
// (tcgen05 TF32/BF16 GEMM, fused triangular solves, the int8 digit split and
// the int8-emulated FP64 GEMM).
#include "common.cuh"
#include "gprat_cu.h"
#include "ozaki.cuh"
#include "tc_gemm.cuh"

#include <algorithm>
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

extern "C" int gprat_cu_test_trsv(int kind, int n, const double *L, const double *b, double *x_fwd, double *x_bwd,
                                  int max_ctas)
{
    try
    {
        if (L == nullptr || b == nullptr || x_fwd == nullptr || x_bwd == nullptr || n <= 0 || (kind != 0 && kind != 1) ||
            max_ctas < 0)
        {
            throw Error(GPRAT_CU_ERR_INVALID_ARG, "gprat_cu_test_trsv: invalid arguments");
        }
        constexpr int B = 128;
        const int nblk = (n + B - 1) / B;
        const int64_t ld = round_up(n, 64);
        // inverses of the diagonal blocks (host, forward substitution per column)
        std::vector<double> inv(static_cast<size_t>(nblk) * B * B, 0.0);
        for (int k = 0; k < nblk; ++k)
        {
            const int r0 = k * B, bs = std::min(B, n - r0);
            double *X = inv.data() + static_cast<size_t>(k) * B * B;
            for (int c = 0; c < bs; ++c)
            {
                for (int r = c; r < bs; ++r)
                {
                    double s = (r == c) ? 1.0 : 0.0;
                    for (int t = c; t < r; ++t)
                    {
                        s -= L[static_cast<int64_t>(r0 + r) * n + r0 + t] * X[t * B + c];
                    }
                    X[r * B + c] = s / L[static_cast<int64_t>(r0 + r) * n + r0 + r];
                }
            }
        }
        const size_t es = kind == 0 ? sizeof(double) : sizeof(float);
        std::vector<char> hL(static_cast<size_t>(n) * ld * es, 0), hI(inv.size() * es, 0);
        for (int r = 0; r < n; ++r)
        {
            for (int c = 0; c <= r; ++c)
            {
                const double v = L[static_cast<int64_t>(r) * n + c];
                if (kind == 0)
                {
                    reinterpret_cast<double *>(hL.data())[static_cast<int64_t>(r) * ld + c] = v;
                }
                else
                {
                    reinterpret_cast<float *>(hL.data())[static_cast<int64_t>(r) * ld + c] = static_cast<float>(v);
                }
            }
        }
        for (size_t q = 0; q < inv.size(); ++q)
        {
            if (kind == 0)
            {
                reinterpret_cast<double *>(hI.data())[q] = inv[q];
            }
            else
            {
                reinterpret_cast<float *>(hI.data())[q] = static_cast<float>(inv[q]);
            }
        }
        Buf dL(hL.size()), dI(hI.size()), dx(n * sizeof(double)), dscr(n * sizeof(double)), dflags(16),
            dStatus(sizeof(DeviceStatus));
        GPRAT_CUDA_CHECK(cudaMemcpy(dL.p, hL.data(), hL.size(), cudaMemcpyHostToDevice));
        GPRAT_CUDA_CHECK(cudaMemcpy(dI.p, hI.data(), hI.size(), cudaMemcpyHostToDevice));
        GPRAT_CUDA_CHECK(cudaMemset(dStatus.p, 0, sizeof(DeviceStatus)));
        cudaStream_t s = nullptr;
        auto *st = static_cast<DeviceStatus *>(dStatus.p);
        auto *x = static_cast<double *>(dx.p);
        for (int dir = 0; dir < 2; ++dir)
        {
            GPRAT_CUDA_CHECK(cudaMemcpy(x, b, n * sizeof(double), cudaMemcpyHostToDevice));
            if (kind == 0)
            {
                const auto *l = static_cast<const double *>(dL.p);
                const auto *li = static_cast<const double *>(dI.p);
                if (dir == 0)
                {
                    trsv_fused_forward(l, ld, li, n, x, static_cast<int *>(dflags.p), static_cast<double *>(dscr.p),
                                       st, s, max_ctas);
                }
                else
                {
                    trsv_fused_backward(l, ld, li, n, x, static_cast<int *>(dflags.p), static_cast<double *>(dscr.p),
                                        st, s, max_ctas);
                }
            }
            else
            {
                const auto *l = static_cast<const float *>(dL.p);
                const auto *li = static_cast<const float *>(dI.p);
                if (dir == 0)
                {
                    trsv_fused_forward_f32(l, ld, li, n, x, static_cast<int *>(dflags.p),
                                           static_cast<double *>(dscr.p), st, s, max_ctas);
                }
                else
                {
                    trsv_fused_backward_f32(l, ld, li, n, x, static_cast<int *>(dflags.p),
                                            static_cast<double *>(dscr.p), st, s, max_ctas);
                }
            }
            GPRAT_CUDA_CHECK(cudaStreamSynchronize(s));
            GPRAT_CUDA_CHECK(cudaMemcpy(dir == 0 ? x_fwd : x_bwd, x, n * sizeof(double), cudaMemcpyDeviceToHost));
        }
        DeviceStatus hst{};
        GPRAT_CUDA_CHECK(cudaMemcpy(&hst, dStatus.p, sizeof(hst), cudaMemcpyDeviceToHost));
        if (hst.timeout != 0)
        {
            throw Error(GPRAT_CU_ERR_TIMEOUT, "triangular solve: a bounded wait timed out");
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

namespace
{

// Digit planes + exponents of one slice operand on the device.
struct OzBuf
{
    Buf dig, exps;
    OzOperand op;
    OzBuf(int rows, int cols, int s, bool block)
        : dig(static_cast<size_t>(s) * round_up(rows, 128) * cols + 128),
          exps(static_cast<size_t>(block ? ceil_div(rows, 128) : rows) * (cols / OZ_KB) * sizeof(int32_t) + 16)
    {
        const int64_t plane = static_cast<int64_t>(round_up(rows, 128)) * cols;
        oz_make_operand(op, static_cast<int8_t *>(dig.p), static_cast<int32_t *>(exps.p), rows, cols, cols, plane,
                        cols / OZ_KB, s, block);
    }
};

}  // namespace

extern "C" int gprat_cu_test_oz_split(int rows, int cols, const double *src, int s, int block, int8_t *digits,
                                      int32_t *exps)
{
    try
    {
        if (src == nullptr || digits == nullptr || exps == nullptr || rows <= 0 || cols <= 0 || cols % OZ_KB != 0 ||
            s < OZ_MIN_SLICES || s > OZ_MAX_SLICES)
        {
            throw Error(GPRAT_CU_ERR_INVALID_ARG, "gprat_cu_test_oz_split: invalid arguments");
        }
        Buf dsrc(static_cast<size_t>(rows) * cols * sizeof(double));
        GPRAT_CUDA_CHECK(cudaMemcpy(dsrc.p, src, static_cast<size_t>(rows) * cols * sizeof(double),
                                    cudaMemcpyHostToDevice));
        OzBuf o(rows, cols, s, block != 0);
        cudaStream_t st = nullptr;
        oz_split(static_cast<const double *>(dsrc.p), cols, rows, cols, block ? nullptr : &o.op,
                 block ? &o.op : nullptr, 0, 0, st);
        GPRAT_CUDA_CHECK(cudaStreamSynchronize(st));
        for (int p = 0; p < s; ++p)
        {
            GPRAT_CUDA_CHECK(cudaMemcpy(digits + static_cast<size_t>(p) * rows * cols,
                                        static_cast<int8_t *>(o.dig.p) + p * o.op.plane,
                                        static_cast<size_t>(rows) * cols, cudaMemcpyDeviceToHost));
        }
        const size_t ne = static_cast<size_t>(block ? ceil_div(rows, 128) : rows) * (cols / OZ_KB);
        GPRAT_CUDA_CHECK(cudaMemcpy(exps, o.exps.p, ne * sizeof(int32_t), cudaMemcpyDeviceToHost));
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

extern "C" int gprat_cu_test_oz_gemm(int M, int N, int K, const double *A, const double *B, double *C, double alpha,
                                     double beta, int lower, int s, int groups, double *rowsq, int max_ctas)
{
    try
    {
        if (A == nullptr || B == nullptr || C == nullptr || M <= 0 || N <= 0 || K <= 0 || K % OZ_KB != 0 ||
            s < OZ_MIN_SLICES || s > OZ_MAX_SLICES || groups < 0 || groups > s || max_ctas < 0)
        {
            throw Error(GPRAT_CU_ERR_INVALID_ARG, "gprat_cu_test_oz_gemm: invalid arguments");
        }
        cudaStream_t st = nullptr;
        const int64_t lc = round_up(N, 2);
        Buf dA(static_cast<size_t>(M) * K * 8), dB(static_cast<size_t>(N) * K * 8), dC(static_cast<size_t>(M) * lc * 8);
        GPRAT_CUDA_CHECK(cudaMemcpy(dA.p, A, static_cast<size_t>(M) * K * 8, cudaMemcpyHostToDevice));
        GPRAT_CUDA_CHECK(cudaMemcpy(dB.p, B, static_cast<size_t>(N) * K * 8, cudaMemcpyHostToDevice));
        GPRAT_CUDA_CHECK(cudaMemcpy2D(dC.p, lc * 8, C, N * 8, N * 8, M, cudaMemcpyHostToDevice));
        OzBuf oa(M, K, s, false), ob(N, K, s, true);
        oz_split(static_cast<const double *>(dA.p), K, M, K, &oa.op, nullptr, 0, 0, st);
        oz_split(static_cast<const double *>(dB.p), K, N, K, nullptr, &ob.op, 0, 0, st);
        Buf dStatus(sizeof(DeviceStatus));
        GPRAT_CUDA_CHECK(cudaMemset(dStatus.p, 0, sizeof(DeviceStatus)));
        Buf dRow(2 * static_cast<size_t>(M) * sizeof(double));
        if (rowsq != nullptr)
        {
            GPRAT_CUDA_CHECK(cudaMemset(dRow.p, 0, 2 * static_cast<size_t>(M) * sizeof(double)));
            GPRAT_CUDA_CHECK(cudaMemcpy(dRow.p, rowsq, M * sizeof(double), cudaMemcpyHostToDevice));
        }
        OzGemmArgs g{};
        g.M = M;
        g.N = N;
        g.K = K;
        g.C = static_cast<double *>(dC.p);
        g.ldc = lc;
        g.alpha = alpha;
        g.beta = beta;
        g.lower = lower != 0;
        g.rowsq = rowsq != nullptr ? static_cast<double *>(dRow.p) : nullptr;
        g.rowsq_half = M;
        g.status = static_cast<DeviceStatus *>(dStatus.p);
        g.max_ctas = max_ctas;
        g.groups = groups;
        oz_gemm(oa.op, ob.op, g, st);
        GPRAT_CUDA_CHECK(cudaStreamSynchronize(st));
        DeviceStatus hs{};
        GPRAT_CUDA_CHECK(cudaMemcpy(&hs, dStatus.p, sizeof(hs), cudaMemcpyDeviceToHost));
        if (hs.timeout != 0)
        {
            throw Error(GPRAT_CU_ERR_TIMEOUT, "int8 GEMM: a bounded wait timed out");
        }
        GPRAT_CUDA_CHECK(cudaMemcpy2D(C, N * 8, dC.p, lc * 8, N * 8, M, cudaMemcpyDeviceToHost));
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

extern "C" int gprat_cu_test_set_wait_budget(int64_t polls)
{
    try
    {
        set_trsv_wait_budget(polls);
        set_last_error("");
        return GPRAT_CU_OK;
    }
    catch (const Error &e)
    {
        set_last_error(e.what());
        return e.code;
    }
}
