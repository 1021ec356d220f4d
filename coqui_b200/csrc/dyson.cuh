// Batched per-(q, iW) Dyson solve for the screened interaction and the RPA log-determinant.
//
// Reference (scr_coulomb_t.cpp:171-199, thc_rpa.icc:130-165) forms A = V Pi, inverts
// I - A by LU and returns W = ([I - V Pi]^{-1} - I) V, and ln det(I - Pi V) by LU.
// Here the Hermitian form of the same quantities is used:
//   V = L L^H (once per q),  M = L^H Pi L,  I - M = C C^H  (FP64 Cholesky),
//   Tr(Pi V) = Tr M,  ln det(I - Pi V) = 2 sum_i ln C_ii,
//   W = L [(I - M)^{-1} - I] L^H = L (D + D^H + D^H D) L^H,  D = C^{-1} - I  (mixed form),
//   W = Y^H Y - V,  Y = C^{-1} L^H  (FP64 form).
#pragma once

#include <cublas_v2.h>
#include <cusolverDn.h>

#include <vector>

#include "common.cuh"

namespace cq {

// In-place lower Cholesky factor (row-major, A = L L^H) of nbatch Np x Np matrices.
// Returns the first nonzero LAPACK info (0 = success).  The strict upper triangle is left
// undefined.
int cholesky_lower_batched(cusolverDnHandle_t sol, double2* A, int64_t Np, int64_t nbatch,
                           cudaStream_t s);

// A[i][j] = conj(A[j][i]) for j > i, nbatch n x n complex64 matrices `stride` elements apart
// (0: n * n).
void launch_mirror_upper(float2* A, int64_t n, int64_t nbatch, cudaStream_t s, int64_t stride = 0);

// Zero the strict upper triangle of L and write LH = L^H (row-major), batched.
void launch_zero_upper_and_adjoint(double2* L, double2* LH, int64_t Np, int64_t nbatch,
                                   cudaStream_t s);

struct DysonArgs {
  int64_t Np = 0, nq = 0, nw = 0;
  const double2* L = nullptr;   // (nq, Np, Np) lower Cholesky factors of V
  const double2* LH = nullptr;  // (nq, Np, Np) L^H
  const double2* V = nullptr;   // (nq, Np, Np)
  const float2* Lc = nullptr;   // mixed form: L and L^H as complex64 tensor-core operands
  const float2* LHc = nullptr;
  bool want_w = true, want_e = false, mixed = true;
  unsigned char* PW = nullptr;  // (nw, nq, Np, Np): Pi(iW) in, W(iW) out (if want_w)
  bool keep_scratch = false;    // use the scratch as it is (a CUDA graph is being captured)
  Prof* prof = nullptr;
  // mixed form: per-problem results on the device (nw * nq entries, n * nq + q); with
  // defer_check the host neither waits nor checks (the caller reads `info` later, e.g. after
  // replaying a captured graph)
  int* info = nullptr;
  double* logdet = nullptr;
  double2* trace = nullptr;
  bool defer_check = false;
};

// Runs every (iW, q) problem; fills logdet / trace (indexed n * nq + q) if want_e.
void dyson_run(const DysonArgs& a, cublasHandle_t blas, cusolverDnHandle_t sol,
               DevBuf<unsigned char>& scratch, cudaStream_t s, std::vector<double>* logdet,
               std::vector<double2>* trace);

}  // namespace cq
