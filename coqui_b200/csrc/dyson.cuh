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

#include <vector>

#include "common.cuh"

namespace cq {

// In-place lower Cholesky factor (row-major, A = L L^H) of nbatch Np x Np matrices on the
// library's FP64 factorisation.  Returns the first nonzero per-problem status (0 = success).
// The strict upper triangle is left as workspace.
int cholesky_lower_batched(double2* A, int64_t Np, int64_t nbatch, cudaStream_t s);

// Lower tile pair (I, J), I >= J, of the 32 x 32 tiling: pair = I (I + 1) / 2 + J.
__device__ __forceinline__ void tile_pair(int pair, int& I, int& J) {
  I = (int)((sqrtf(8.f * (float)pair + 1.f) - 1.f) * 0.5f);
  while ((I + 1) * (I + 2) / 2 <= pair) ++I;
  while (I > 0 && I * (I + 1) / 2 > pair) --I;
  J = pair - I * (I + 1) / 2;
}

// E = DH + DH^H + F (n x n complex64, row-major; only the lower triangle i >= j of the
// Hermitian F is read) on the tile pair (I, J), I >= J, by a CTA of 256 threads: DH(I, J),
// DH(J, I) and F(I, J) are loaded in one round, E(I, J) and its adjoint E(J, I) written.
__device__ __forceinline__ void herm_sum_pair(const float2* __restrict__ d,
                                              const float2* __restrict__ fp,
                                              float2* __restrict__ e, int64_t n, int I, int J) {
  __shared__ float2 a[32][33];  // DH(I, J)
  __shared__ float2 b[32][33];  // DH(J, I)
  __shared__ float2 f[32][33];  // F(I, J) on and below the diagonal
  const int64_t i0 = (int64_t)I * 32, j0 = (int64_t)J * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const float2 z = make_float2(0.f, 0.f);
  for (int r = ty; r < 32; r += 8) {
    const int64_t gi = i0 + r, gj = j0 + tx;  // tile (I, J)
    const int64_t hi = j0 + r, hj = i0 + tx;  // tile (J, I)
    const bool in = gi < n && gj < n;
    a[r][tx] = in ? d[gi * n + gj] : z;
    b[r][tx] = (hi < n && hj < n) ? d[hi * n + hj] : z;
    f[r][tx] = (in && gi >= gj) ? fp[gi * n + gj] : z;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    // E[i][j] = DH[i][j] + conj(DH[j][i]) + F[i][j], F[i][j] = conj(F[j][i]) above the diagonal
    const int64_t gi = i0 + r, gj = j0 + tx;
    float2 fv = f[r][tx];
    if (gi < gj) fv = make_float2(f[tx][r].x, -f[tx][r].y);  // diagonal tile only
    const float2 x = a[r][tx], y = b[tx][r];
    if (gi < n && gj < n) e[gi * n + gj] = make_float2(x.x + y.x + fv.x, x.y - y.y + fv.y);
  }
  if (I != J) {
    for (int r = ty; r < 32; r += 8) {
      // E[j0 + r][i0 + tx] = conj(E[i0 + tx][j0 + r])
      const int64_t gi = j0 + r, gj = i0 + tx;
      const float2 x = a[tx][r], y = b[r][tx], t = f[tx][r];
      if (gi < n && gj < n) e[gi * n + gj] = make_float2(x.x + y.x + t.x, -x.y + y.y - t.y);
    }
  }
}

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

// Free device memory (bytes, beside the scratch it already holds) with which dyson_run
// forms chunks of two whole waves of the factorisation (or all nprob problems) for the W step.
size_t dyson_reserve_bytes(int64_t Np, int64_t nprob, bool mixed);

// Runs every (iW, q) problem; fills logdet / trace (indexed n * nq + q) if want_e.
void dyson_run(const DysonArgs& a, DevBuf<unsigned char>& scratch, cudaStream_t s,
               std::vector<double>* logdet, std::vector<double2>* trace);

}  // namespace cq
