// Batched complex GEMMs of the mixed-precision path (projections and Dyson products).
#pragma once

#include "common.cuh"

namespace cq {

// THC collocation X (nk, Np, nb) prepared for the projection GEMMs.
struct TcOperand {
  const double2* X = nullptr;
  int64_t nk = 0, Np = 0, nb = 0;
  DevBuf<unsigned char> packed;  // X^T per k (nk, nb, Np), complex128
  DevBuf<unsigned char> tmp;     // per-call intermediate (X G or S X)
  void release() {
    packed.release();
    tmp.release();
  }
};

void tc_pack_X(TcOperand& op, const double2* X, int64_t nk, int64_t Np, int64_t nb,
               cudaStream_t s);

// out[k] = X^k G^k X^k^H  (Np x Np, complex64), G (nk, nb, nb) complex128.
void tc_project_p2a(TcOperand& op, const double2* Gk, float2* out, int64_t nk, int64_t Np,
                    int64_t nb, cudaStream_t s);

// out[k] = X^k^H S^k X^k  (nb x nb, complex128), S (nk, Np, Np) complex64.
void tc_project_a2p(TcOperand& op, const float2* Sk, double2* out, int64_t nk, int64_t Np,
                    int64_t nb, cudaStream_t s);

// Split-TF32 tensor-core GEMM, "NT" form:
//   C[b](m, n) = sum_k opA(A[b])(m, k) * opB(Bt[b])(n, k)
// A: row-major M x K (lda), Bt: row-major N x K (ldb), each complex64 or complex128
// (the *_c128 flags) and optionally conjugated; C: row-major complex64 (ldc).  Strides in
// complex elements; sA/sB/sC are the batch strides.
void tc_cgemm_nt(const void* A, bool a_c128, bool conj_a, int64_t lda, int64_t sA, const void* Bt,
                 bool b_c128, bool conj_b, int64_t ldb, int64_t sB, float2* C, int64_t ldc,
                 int64_t sC, int64_t M, int64_t N, int64_t K, int64_t batch, cudaStream_t s);

// Returns (and clears) the device flag set when a bounded wait inside a tensor-core kernel
// gave up (nonzero = a kernel timed out).
int tc_take_error();

}  // namespace cq
