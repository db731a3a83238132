// int8 split-precision complex GEMM on tcgen05 (see gemm_i8.cu).
#pragma once
#include "imps_internal.h"

namespace imps {

// One operand cut into `s` int8 planes (K-major, padded), plus per-line scales.
struct SplitOperand {
  DevBuf data;    // s planes of Rp x Kp bytes
  DevBuf scale;   // per complex row (A side) / column (B side): power of two > max |re|,|im|
  DevBuf inv;     // 1 / scale
  DevBuf mx;      // scratch for the max reduction
  int rows = 0;   // complex rows (A: M, B: N)
  int K = 0;      // complex inner dimension
  int s = 0;      // slices stored
  int64_t Rp = 0, Kp = 0;
};

// op(A) (M x K), op in {N, C}: expanded real rows (2M) x (2K) int8 planes
void split_operand_a(Context* ctx, SplitOperand& S, Op op, int M, int K, const dcplx* A, int64_t lda, int s);
// op(B) (K x N), op in {N, C}: N rows x (2K) int8 planes
void split_operand_b(Context* ctx, SplitOperand& S, Op op, int K, int N, const dcplx* B, int64_t ldb, int s);
// C (complex, ldc) = alpha * op(A) op(B) (+ C when accumulate) using `s` slice diagonals
void split_gemm(Context* ctx, const SplitOperand& A, const SplitOperand& B, int s, double alpha, bool accumulate,
                dcplx* C, int64_t ldc);

// Slices needed for a requested relative accuracy `tol` (clamped to 2..8).
int slices_for_tol(double tol);

}  // namespace imps
