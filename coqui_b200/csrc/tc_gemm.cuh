// Batched complex GEMMs of the mixed-precision path (projections and Dyson products).
#pragma once

#include "common.cuh"

namespace cq {

enum class TcOp { N, C };  // C = conjugate transpose

// THC collocation X (nk, Np, nb) prepared for the projection GEMMs.
struct TcOperand {
  const double2* X = nullptr;
  int64_t nk = 0, Np = 0, nb = 0;
  DevBuf<unsigned char> packed;  // packed operand planes
  DevBuf<unsigned char> tmp;     // per-call intermediate (X G or X^H S)
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

// C[b] = opA(A[b]) opB(B[b]) (- C[b] if minus_c), row-major, batch strides M*K, K*N, M*N.
template <typename TA, typename TB>
void tc_gemm_c(TcOp opa, const TA* A, TcOp opb, const TB* B, float2* C, int64_t M, int64_t N,
               int64_t K, int64_t batch, cudaStream_t s, bool minus_c = false);

}  // namespace cq
