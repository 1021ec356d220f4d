// Batched FP64 Cholesky / log-determinant / triangular inverse of A = I - M.
#pragma once

#include "common.cuh"

namespace cq {

// For each of nprob Np x Np problems: A = I - M (lower triangle of M, complex64, is read),
// A <- C with A = C C^H (FP64, lower), logdet = 2 sum ln C_ii, trace = sum M_ii,
// info = 1 if a pivot was not positive.  If Z is non-null: Z <- C^{-H} - I (upper; computed
// in FP64, stored as complex64).  A's upper triangle is used as FP64 workspace.
void launch_chol_inv(const float2* M, double2* A, float2* Z, double* logdet, double2* trace,
                     int* info, int64_t Np, int64_t nprob, cudaStream_t s);

// One problem of a grouped factorisation: M (n x n complex64, lower triangle read), A (n x n
// FP64 workspace, C and C^{-H} on return), Z (n x n complex64, C^{-H} - I written).
struct CholProblem {
  const float2* M;
  double2* A;
  float2* Z;
  int64_t n;
};

// Diagonal group edge of the FP64 inverse when the tensor cores form the off-group blocks.
constexpr int64_t kInvGroup = 128;

// launch_chol_inv with Z for problems of different sizes in one launch per step (prep,
// factorisation + full FP64 inverse, Z); results per problem in table order.  With
// group_inverse the inverse is formed only inside the kInvGroup diagonal groups (as
// launch_chol_group_inv) and Z is not written: launch_chol_split and the tensor-core levels
// take over.
void launch_chol_inv_grouped(const std::vector<CholProblem>& probs, DevBuf<unsigned char>& table,
                             double* logdet, double2* trace, int* info, cudaStream_t s,
                             bool group_inverse = false);

// The same results as launch_chol_inv_grouped(..., group_inverse = true) with each problem
// spread over many CTAs: one launch per phase of every block column (the diagonal block; the
// panel blocks below it; the trailing blocks), then one for the group inverse.  Problems of
// equal size must be consecutive (at most 64 runs).  For sets whose largest problem would
// otherwise set the finishing time (few problems, or a few much larger than the rest).
void launch_chol_tiled(const std::vector<CholProblem>& probs, DevBuf<unsigned char>& table,
                       double* logdet, double2* trace, int* info, cudaStream_t s);
// launch_chol_group_inv through the tiled path (problems at M + p Np^2, A + p Np^2)
void launch_chol_tiled_strided(const float2* M, double2* A, double* logdet, double2* trace,
                               int* info, int64_t Np, int64_t nprob, cudaStream_t s);
// Whether the tiled path finishes sooner for problems of these sizes (one CTA per problem
// leaves the GPU mostly idle while the largest problem finishes); the environment variable
// COQUI_B200_CHOL_TILED=1 or 0 forces the choice.
bool chol_prefer_tiled(const std::vector<int64_t>& sizes);

// FP64 form: A = I - M with M complex128 (lower triangle read), A <- C (lower, FP64), the
// whole inverse C^{-H} in the upper triangle, logdet, trace, info per problem (four-warp
// kernel, same arithmetic as the complex64 form).
void launch_chol_inv_c128(const double2* M, double2* A, double* logdet, double2* trace, int* info,
                          int64_t Np, int64_t nprob, cudaStream_t s);
// Z = U - I from the upper triangle U of A, zero below the diagonal (complex128, batched).
void launch_upper_minus_eye(const double2* A, double2* Z, int64_t Np, int64_t nprob,
                            cudaStream_t s);

// Problems one launch of the one-CTA factorisation (launch_chol_group_inv) runs at once on
// the current device: SMs x resident CTAs per SM.  A batch of a multiple of this size leaves
// no partly filled last wave.
int64_t chol_wave_size();

// As launch_chol_inv without Z, but the inverse U = C^{-H} is formed only inside the
// kInvGroup x kInvGroup diagonal groups (upper triangle of A there).
void launch_chol_group_inv(const float2* M, double2* A, double* logdet, double2* trace, int* info,
                           int64_t Np, int64_t nprob, cudaStream_t s);

// Complex64 operands of the tensor-core inverse levels (all Np x Np per problem):
// Z = U - I (group upper triangles; 0 below the diagonal), Zl = U^H - I (group lower
// triangles; 0 elsewhere), Zc = -C (strictly lower off-group blocks only).
void launch_chol_split(const double2* A, float2* Z, float2* Zl, float2* Zc, int64_t Np,
                       int64_t nprob, cudaStream_t s);

// Zl[r1 + c][r0 + r] = conj(Z[r0 + r][r1 + c]), r < b, c < b1.
void launch_block_adjoint(const float2* Z, float2* Zl, int64_t Np, int64_t r0, int64_t r1,
                          int64_t b, int64_t b1, int64_t nprob, cudaStream_t s);

}  // namespace cq
