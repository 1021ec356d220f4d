// Batched complex128 GEMM on the FP64 tensor cores (DMMA), row-major operands:
//   C[b] = alpha op(A[b]) op(B[b]) + beta C[b],  op = 'N' (as stored) or 'C' (conjugate
//   transpose), op(A) M x K, op(B) K x N.
// Batches are strided (stride 0 broadcasts one operand) or given as device arrays of per-
// problem pointers.  Known triangular structure of op(A) / op(B) trims each tile's K range,
// and lower_only skips the tiles strictly above the diagonal (their C is left as it was).
#pragma once

#include "common.cuh"

namespace cq {

struct ZgemmArgs {
  char opA = 'N', opB = 'N';
  int64_t M = 0, N = 0, K = 0;
  double2 alpha = {1.0, 0.0}, beta = {0.0, 0.0};
  const double2* A = nullptr;
  int64_t lda = 0, sA = 0;
  const double2* B = nullptr;
  int64_t ldb = 0, sB = 0;
  double2* C = nullptr;
  int64_t ldc = 0, sC = 0;
  int64_t batch = 1;
  // pointer-array form (device arrays of batch pointers) when Ap is set
  const double2* const* Ap = nullptr;
  const double2* const* Bp = nullptr;
  double2* const* Cp = nullptr;
  // structure: op(A) upper (k >= m) / lower (k <= m) triangular, op(B) lower (k >= n) /
  // upper (k <= n) triangular; lower_only: only tiles on or below the diagonal are formed
  bool a_upper = false, a_lower = false, b_lower = false, b_upper = false, lower_only = false;
  // upper_zero: tiles strictly below the diagonal are written as zeros without products
  bool upper_zero = false;
  // periodic batch index of A / B (0 = off): problem b uses operand (q0 + b) % mod, for
  // per-q operands of problems ordered (frequency, q)
  int64_t a_mod = 0, a_q0 = 0, b_mod = 0, b_q0 = 0;
};

void zgemm(const ZgemmArgs& a, cudaStream_t s);

}  // namespace cq
