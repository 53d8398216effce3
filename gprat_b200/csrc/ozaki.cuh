// FP64 matrix products on the int8 tensor cores (Ozaki scheme).
//
// Method: K. Ozaki, T. Ogita, S. Oishi, S. M. Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix
// multiplication and its applications", Numer. Algorithms 59 (2012) 95-118,
// in the integer form of H. Ootomo, K. Ozaki, R. Yokota, "DGEMM on integer
// matrix multiplication unit", IJHPCA 38 (2024).
//
// A row-major FP64 matrix X is held as s int8 digit planes D_0..D_{s-1}
// and power-of-two scales ("slices"):
//     X[r][c] ~= 2^(e - 6) * sum_{p < s} D_p[r][c] * 254^(-p),
//     |D_0| <= 64, |D_p| <= 127 (p >= 1),
// with one exponent e per row and 128-column block ("row" operand) or per
// 128 x 128 block ("block" operand); |X| < 2^e over the exponent's domain,
// so the representation keeps 6 + 7.99 (s - 1) bits relative to that
// maximum (base 254 is the largest whose balanced digits fit int8).
// A product C = A B^T over one 128-column block k is then
//     2^(eA + eB - 12) * sum_{g < G} 254^(-g) * P_g,
//     P_g = sum_{p + q = g} D^A_p (D^B_q)^T          (exact in int32)
// and the G = s groups of one block form one unit of int32 accumulation in
// tensor memory (tcgen05.mma kind::i8) each; the epilogue combines two
// groups exactly in int32 (254 P_g + P_{g+1}, at most 2,112,012,032 for
// the largest pair (4, 5)), converts the sum exactly to FP64 and adds it
// with its scale by one FMA, so the roundings are the digit truncation, the
// scale 254^-(g+1) and FP64 additions.
#pragma once

#include "common.cuh"

#include <cuda.h>

namespace gprat_cu
{

constexpr int OZ_KB = 128;  // columns per exponent block = digit bytes per TMA box row
constexpr int OZ_MIN_SLICES = 3;
constexpr double OZ_BASE = 254.0;  // digit base
constexpr int OZ_IBASE = 254;
constexpr int OZ_MAX_SLICES = 7;

struct OzOperand
{
    int8_t *digits = nullptr;  // plane p, row r, column c at digits + p * plane + r * ld + c
    int32_t *exps = nullptr;   // row operand: exps[r * ldE + c / 128]; block operand: exps[(r / 128) * ldE + c / 128]
    int rows = 0, cols = 0;    // cols a multiple of 128
    int64_t ld = 0;            // bytes per digit row (a multiple of 128)
    int64_t plane = 0;         // bytes per digit plane (>= rows * ld)
    int ldE = 0;               // exponent row stride (>= cols / 128)
    int s = 0;                 // digit planes
    bool block = false;        // block exponents (B role) instead of row exponents (A role)
    CUtensorMap map_a;         // TMA map, box 128 bytes x 128 rows x 1 plane (A role)
    CUtensorMap map_b;         // TMA map, box 128 bytes x 64 rows x 1 plane (B role, one CTA's half)
};

// Describes (and builds the TMA maps of) a slice operand over caller-owned
// buffers: digits (16-byte aligned, s planes of `plane` bytes), exps.
void oz_make_operand(OzOperand &op, int8_t *digits, int32_t *exps, int rows, int cols, int64_t ld, int64_t plane,
                     int ldE, int s, bool block);

// Splits src (rows x cols FP64, row-major, lds; cols a multiple of 128) into
// the digits and exponents of row_op and/or blk_op (either may be null) at
// (dst_row0, dst_col0) of those operands.  dst_col0 must be a multiple of
// 128; for blk_op, dst_row0 too (block exponents cover 128-row blocks of the
// destination, taken over the rows < rows of each block).
void oz_split(const double *src, int64_t lds, int rows, int cols, const OzOperand *row_op, const OzOperand *blk_op,
              int dst_row0, int dst_col0, cudaStream_t s);

struct OzGemmArgs
{
    int M, N, K;         // K a multiple of 128
    int a_row0, a_col0;  // origin of A in its (row) operand; a_col0 a multiple of 128
    int b_row0, b_col0;  // origin of B in its (block) operand; both multiples of 128
    double *C;           // FP64, 16-byte aligned, ldc even
    int64_t ldc;
    double alpha, beta;  // beta 0 or 1
    bool lower;          // M == N; only C[i][j] with i >= j is written
    // optional (beta = 0, not lower): rowsq[h * rowsq_half + i] += sum over
    // the columns of half h (j < 64 or j >= 64 of each 128-column tile) of
    // C_new[i][j]^2; one writer per word and launch (deterministic)
    double *rowsq;
    int64_t rowsq_half;
    DeviceStatus *status;  // timeout flag if a bounded wait gives up
    int max_ctas;          // persistent grid bound (0 = every SM), leaves SMs to other streams
    int groups;            // digit groups kept, 1..s (0 = s)
};

// C = beta C + alpha A B^T, A = rows [a_row0, a_row0 + M) of a row operand,
// B = rows [b_row0, b_row0 + N) of a block operand (same s), columns from
// a_col0 / b_col0 on for K.  Tiles of 256 x 128 on CTA pairs
// (tcgen05.mma.cta_group::2.kind::i8).
void oz_gemm(const OzOperand &A, const OzOperand &B, const OzGemmArgs &args, cudaStream_t s);

}  // namespace gprat_cu
