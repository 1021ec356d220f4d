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

}  // namespace cq
