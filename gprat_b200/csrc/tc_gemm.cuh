// Host-side interface of the tcgen05 (5th-generation tensor core) GEMM used
// by the mixed-precision path:  C[MxN] (FP32) = beta*C + alpha * A B^T,
// A (M x K) and B (N x K) K-contiguous in global memory as FP32 (TF32 MMA)
// or BF16, staged by TMA, accumulated in FP32 in tensor memory.
#pragma once

#include "common.cuh"

#include <cuda.h>

namespace gprat_cu
{

enum class TcKind : int
{
    TF32 = 0,  // FP32 operands, tcgen05.mma kind::tf32
    BF16 = 1,  // BF16 operands, tcgen05.mma kind::f16 (bf16 inputs)
};

// A 2-D row-major operand matrix (rows x cols, leading dimension ld
// elements) described by a TMA tensor map with a 128-row x 128-byte box and
// 128-byte swizzle.
struct TcOperand
{
    CUtensorMap map;
    const void *base = nullptr;
    int rows = 0, cols = 0;
    int64_t ld = 0;
    TcKind kind = TcKind::TF32;
};

// Builds the tensor map (base must be 16-byte aligned, ld*element size a
// multiple of 16 bytes).
void tc_make_operand(TcOperand &op, const void *base, int rows, int cols, int64_t ld, TcKind kind);

struct TcGemmArgs
{
    int M, N, K;      // K must be a multiple of the 128-byte stage depth (32 TF32 / 64 BF16 elements)
    int a_row0, a_col0;  // origin of A inside its operand matrix
    int b_row0, b_col0;  // origin of B inside its operand matrix
    float *C;
    int64_t ldc;
    float alpha, beta;  // beta must be 0 or 1
    bool lower;         // M == N; only C[i][j] with i >= j is updated, tiles above the diagonal skipped
                        // (within diagonal tiles, beta = 0 writes 0 above the diagonal)
    // optional (N <= 128, beta = 0): per-row sums of squares of the new C, split by
    // column half so that no two threads add into one word (deterministic):
    // rowsq[i] += sum_{j<64} C_new[i][j]^2, rowsq[rowsq_half + i] += sum_{j>=64} ...
    double *rowsq;
    int64_t rowsq_half;  // >= M when rowsq is set
    DeviceStatus *status;  // receives the timeout flag if a bounded wait gives up
    int max_ctas;          // persistent grid limit (0 = one CTA per SM); leaves SMs to concurrent streams
    int tile_mode;         // 0 = automatic; 1 = 128 x 128, 2 = 128 x 256, 3 = 256 x 256 on a CTA pair (tests)
};

void tc_gemm(const TcOperand &A, const TcOperand &B, const TcGemmArgs &args, cudaStream_t s);

// Element-wise conversions used around the tensor-core kernels.
void convert_f64_to_f32(const double *src, int64_t lds, float *dst, int64_t ldd, int rows, int cols, cudaStream_t s);
void convert_f32_to_f64(const float *src, int64_t lds, double *dst, int64_t ldd, int rows, int cols, cudaStream_t s);
void convert_f32_to_bf16(const float *src, int64_t lds, void *dst, int64_t ldd, int rows, int cols, cudaStream_t s);

}  // namespace gprat_cu
