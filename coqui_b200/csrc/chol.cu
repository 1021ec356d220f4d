// Batched FP64 Cholesky factorisation, log-determinant and triangular inverse of
// A = I - M (one CTA per Np x Np problem), the factorisation step of the Dyson solve.
//
//   A = C C^H (C lower, FP64), logdet = 2 sum_i ln C_ii, trace = sum_i M_ii,
//   optional DH = C^{-H} - I (upper triangular, FP64) for W = L (D + D^H + D^H D) L^H.
//
// Right-looking blocked algorithm with 32 x 32 blocks: the diagonal block is factored and
// inverted in shared memory, the panel below is L_ib = A_ib C_jj^{-H}, the trailing lower
// triangle gets A_ik -= L_ij L_kj^H.  The inverse is formed block column by block column:
// X_ij = -C_ii^{-1} sum_{k=j}^{i-1} C_ik X_kj.  Block products use 4 x 4 register tiles per
// thread (64 threads per 32 x 32 output), operands staged in shared memory; ~50 KB of
// shared memory per problem lets four problems share an SM so that one problem's barriers
// and loads overlap another's FP64 arithmetic.  A = I - M is set up and D^H written out by
// separate element-wise kernels.
#include <cstdint>

#include "chol.cuh"

namespace cq {

namespace {

constexpr int CB = 32;       // block size
constexpr int CT = 64;       // threads per CTA
constexpr int TW = 8;        // thread grid edge: (TW x TW) threads x (4 x 4) outputs = CB x CB
constexpr int PITCH = CB + 1;  // smem row pitch (double2 elements)

__device__ __forceinline__ double2 cmul_(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc_(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 conj_(double2 a) { return make_double2(a.x, -a.y); }

// smem tile <- global block (rows r0.., cols c0..) of an ld x ld row-major matrix, rb x cb valid
__device__ __forceinline__ void load_blk(double2* S, const double2* G, int64_t ld, int64_t r0,
                                         int64_t c0, int rb, int cb) {
  double2 v[CB * CB / CT];
#pragma unroll
  for (int u = 0; u < CB * CB / CT; ++u) {  // all loads in flight before the smem stores
    const int i = threadIdx.x + u * CT;
    const int r = i / CB, c = i % CB;
    v[u] = (r < rb && c < cb) ? G[(r0 + r) * ld + c0 + c] : make_double2(0, 0);
  }
#pragma unroll
  for (int u = 0; u < CB * CB / CT; ++u) {
    const int i = threadIdx.x + u * CT;
    S[(i / CB) * PITCH + i % CB] = v[u];
  }
}
// smem tile <- conj transpose of a global block: S[r][c] = conj(G[c0 + c][r0 + r])... given as
// (the block stored at rows gr0, cols gc0 with gr x gc valid) -> S = G_blk^H
__device__ __forceinline__ void load_blk_adj(double2* S, const double2* G, int64_t ld, int64_t gr0,
                                             int64_t gc0, int gr, int gc) {
  double2 v[CB * CB / CT];
#pragma unroll
  for (int u = 0; u < CB * CB / CT; ++u) {
    const int i = threadIdx.x + u * CT;
    const int r = i / CB, c = i % CB;  // S[c][r] = conj(G[gr0 + r][gc0 + c])
    v[u] = (r < gr && c < gc) ? conj_(G[(gr0 + r) * ld + gc0 + c]) : make_double2(0, 0);
  }
#pragma unroll
  for (int u = 0; u < CB * CB / CT; ++u) {
    const int i = threadIdx.x + u * CT;
    S[(i % CB) * PITCH + i / CB] = v[u];
  }
}
// S (lower triangular part) <- adjoint of the upper triangle of a global diagonal block:
// S[r][c] = conj(G[r0 + c][r0 + r]) for r >= c, 0 above
__device__ __forceinline__ void load_blk_adjU(double2* S, const double2* G, int64_t ld, int64_t r0,
                                              int nb) {
  double2 v[CB * CB / CT];
#pragma unroll
  for (int u = 0; u < CB * CB / CT; ++u) {
    const int i = threadIdx.x + u * CT;
    const int r = i / CB, c = i % CB;  // v = conj(G[r0 + r][r0 + c]) feeds S[c][r], c >= r
    v[u] = (r < nb && c < nb && c >= r) ? conj_(G[(r0 + r) * ld + r0 + c]) : make_double2(0, 0);
  }
#pragma unroll
  for (int u = 0; u < CB * CB / CT; ++u) {
    const int i = threadIdx.x + u * CT;
    S[(i % CB) * PITCH + i / CB] = v[u];
  }
}
// upper triangle of a global diagonal block <- adjoint of the lower-triangular S:
// G[r0 + c][r0 + r] = conj(S[r][c]) for r >= c
__device__ __forceinline__ void store_blk_adjU(const double2* S, double2* G, int64_t ld, int64_t r0,
                                               int nb) {
#pragma unroll
  for (int u = 0; u < CB * CB / CT; ++u) {
    const int i = threadIdx.x + u * CT;
    const int r = i / CB, c = i % CB;
    if (r < nb && c < nb && r >= c) G[(r0 + c) * ld + r0 + r] = conj_(S[r * PITCH + c]);
  }
}
__device__ __forceinline__ void store_blk(const double2* S, double2* G, int64_t ld, int64_t r0,
                                          int64_t c0, int rb, int cb) {
#pragma unroll
  for (int u = 0; u < CB * CB / CT; ++u) {
    const int i = threadIdx.x + u * CT;
    const int r = i / CB, c = i % CB;
    if (r < rb && c < cb) G[(r0 + r) * ld + c0 + c] = S[r * PITCH + c];
  }
}

// acc[i][j] (rows ty + TW i, cols tx + TW j) += sum_k X[r][k] * Y'[k][c] over k < K, where
// Y'(k, c) = conj(Y[c][k]) if ADJ_Y (product with Y^H) else Y[k][c].
template <bool ADJ_Y>
__device__ __forceinline__ void mma_tile(const double2* X, const double2* Y, int K,
                                         double2 (&acc)[4][4]) {
  const int tx = threadIdx.x % TW, ty = threadIdx.x / TW;
  for (int k = 0; k < K; ++k) {
    double2 a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = X[(ty + TW * i) * PITCH + k];
#pragma unroll
    for (int j = 0; j < 4; ++j)
      b[j] = ADJ_Y ? conj_(Y[(tx + TW * j) * PITCH + k]) : Y[k * PITCH + tx + TW * j];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        acc[i][j].x = fma(a[i].x, b[j].x, fma(-a[i].y, b[j].y, acc[i][j].x));
        acc[i][j].y = fma(a[i].x, b[j].y, fma(a[i].y, b[j].x, acc[i][j].y));
      }
  }
}

// acc[i][j] -= sum_k X[r][k] conj(Y[c][k])  (A - X Y^H)
__device__ __forceinline__ void mma_tile_sub(const double2* X, const double2* Y, int K,
                                             double2 (&acc)[4][4]) {
  const int tx = threadIdx.x % TW, ty = threadIdx.x / TW;
  for (int k = 0; k < K; ++k) {
    double2 a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = X[(ty + TW * i) * PITCH + k];
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = Y[(tx + TW * j) * PITCH + k];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        // a * conj(b) = (ax bx + ay by) + i (ay bx - ax by)
        acc[i][j].x = fma(-a[i].x, b[j].x, fma(-a[i].y, b[j].y, acc[i][j].x));
        acc[i][j].y = fma(-a[i].y, b[j].x, fma(a[i].x, b[j].y, acc[i][j].y));
      }
  }
}

__device__ __forceinline__ void zero_acc(double2 (&acc)[4][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0, 0);
}

// In-place Cholesky of the lower triangle of S (n x n); adds sum ln C_ii to *ld_acc
// (thread 0) and sets *bad if a pivot is not positive.  One barrier per column: column c is
// used unscaled (times 1/d_c) in its rank-1 update and scaled during the next column's step.
__device__ void factor_diag(double2* S, int n, double* ld_acc, int* bad) {
  double prev_inv = 1.0, prev_d = 1.0;
  for (int c = 0; c < n; ++c) {
    __syncthreads();
    double d = S[c * PITCH + c].x;
    const bool good = d > 0.0;
    d = good ? sqrt(d) : 1.0;
    const double inv = 1.0 / d;
    if (c > 0) {  // finish column c - 1: diagonal and scaled entries below it
      if (threadIdx.x == 0) S[(c - 1) * PITCH + c - 1] = make_double2(prev_d, 0.0);
      for (int r = c + threadIdx.x; r < n; r += CT) {
        S[r * PITCH + c - 1].x *= prev_inv;
        S[r * PITCH + c - 1].y *= prev_inv;
      }
    }
    const int m = n - c - 1;
    const double inv2 = inv * inv;
    for (int idx = threadIdx.x; idx < m * m; idx += CT) {
      const int r = c + 1 + idx / m, s = c + 1 + idx % m;
      if (s <= r) {
        const double2 u = cmulc_(S[r * PITCH + c], S[s * PITCH + c]);
        S[r * PITCH + s].x -= u.x * inv2;
        S[r * PITCH + s].y -= u.y * inv2;
      }
    }
    if (threadIdx.x == 0) {
      if (!good) *bad = 1;
      *ld_acc += log(d);
    }
    prev_inv = inv;
    prev_d = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) S[(n - 1) * PITCH + n - 1] = make_double2(prev_d, 0.0);
  __syncthreads();
}

// Sinv = inverse of the lower-triangular S (n x n): forward substitution with one column
// per pair of lanes (partial dot products reduced by a shuffle).
__device__ void invert_lower(const double2* S, double2* Sinv, int n) {
  for (int i = threadIdx.x; i < CB * CB; i += CT) Sinv[(i / CB) * PITCH + i % CB] = make_double2(0, 0);
  __syncthreads();
  const int c = threadIdx.x >> 1, sub = threadIdx.x & 1;
  const bool col = c < n;
  if (col && sub == 0) Sinv[c * PITCH + c] = make_double2(1.0 / S[c * PITCH + c].x, 0.0);
  __syncwarp();
  for (int r = 1; r < n; ++r) {
    double ax = 0, ay = 0;
    if (col && r > c)
      for (int k = c + sub; k < r; k += 2) {
        const double2 u = cmul_(S[r * PITCH + k], Sinv[k * PITCH + c]);
        ax += u.x;
        ay += u.y;
      }
    ax += __shfl_xor_sync(0xffffffffu, ax, 1);
    ay += __shfl_xor_sync(0xffffffffu, ay, 1);
    if (col && r > c && sub == 0) {
      const double inv = -1.0 / S[r * PITCH + r].x;
      Sinv[r * PITCH + c] = make_double2(ax * inv, ay * inv);
    }
    __syncwarp();
  }
  __syncthreads();
}

// inv_group: the inverse is formed within diagonal groups of inv_group blocks only (the
// whole matrix when inv_group >= nblk); the tensor-core levels fill in the rest.
// One problem: M, A (n x n), results at logdet/trace/info[0].
template <bool INV>
__device__ __forceinline__ void chol_inv_problem(const float2* __restrict__ M,
                                                 double2* __restrict__ A,
                                                 double* __restrict__ logdet,
                                                 double2* __restrict__ trace,
                                                 int* __restrict__ info, int64_t n, int inv_group) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* S0 = reinterpret_cast<double2*>(smem_raw);
  double2* S1 = S0 + CB * PITCH;
  double2* S2 = S1 + CB * PITCH;
  __shared__ double s_ld;
  __shared__ int s_bad;
  __shared__ double s_red[2][CT];
  const int nblk = (int)((n + CB - 1) / CB);
  const int tx = threadIdx.x % TW, ty = threadIdx.x / TW;

  if (threadIdx.x == 0) {
    s_ld = 0.0;
    s_bad = 0;
  }
  // trace of M (A = I - M was set up by k_chol_prep)
  double tr = 0, ti = 0;
  for (int64_t i = threadIdx.x; i < n; i += CT) {
    const float2 m = M[i * n + i];
    tr += m.x;
    ti += m.y;
  }
  s_red[0][threadIdx.x] = tr;
  s_red[1][threadIdx.x] = ti;
  __syncthreads();

  for (int j = 0; j < nblk; ++j) {
    const int64_t j0 = (int64_t)j * CB;
    const int jb = (int)(CB < (n - j0) ? (int64_t)CB : (n - j0));
    // 1. diagonal block: factor and invert
    load_blk(S0, A, n, j0, j0, jb, jb);
    __syncthreads();
    factor_diag(S0, jb, &s_ld, &s_bad);
    invert_lower(S0, S1, jb);
    // C_jj is not needed again; the upper triangle of the diagonal block keeps C_jj^{-H}
    if (INV) store_blk_adjU(S1, A, n, j0, jb);
    __syncthreads();
    // 2. panel: L_ib = A_ib C_jj^{-H}
    for (int ib = j + 1; ib < nblk; ++ib) {
      const int64_t i0 = (int64_t)ib * CB;
      const int rb = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
      load_blk(S2, A, n, i0, j0, rb, jb);
      __syncthreads();
      double2 acc[4][4];
      zero_acc(acc);
      mma_tile<true>(S2, S1, jb, acc);
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int r = ty + TW * i, c = tx + TW * jj;
          if (r < rb && c < jb) A[(i0 + r) * n + j0 + c] = acc[i][jj];
        }
      __syncthreads();
    }
    // 3. trailing update of the lower triangle: A_ik -= L_ij L_kj^H
    for (int kb = j + 1; kb < nblk; ++kb) {
      const int64_t k0 = (int64_t)kb * CB;
      const int kbsz = (int)(CB < (n - k0) ? (int64_t)CB : (n - k0));
      load_blk(S0, A, n, k0, j0, kbsz, jb);
      for (int ib = kb; ib < nblk; ++ib) {
        const int64_t i0 = (int64_t)ib * CB;
        const int rb = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
        load_blk(S2, A, n, i0, j0, rb, jb);
        __syncthreads();
        double2 acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)  // start from the current A block (loads in flight early)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const int r = ty + TW * i, c = tx + TW * jj;
            acc[i][jj] = (r < rb && c < kbsz && (ib > kb || c <= r)) ? A[(i0 + r) * n + k0 + c]
                                                                      : make_double2(0, 0);
          }
        mma_tile_sub(S2, S0, jb, acc);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const int r = ty + TW * i, c = tx + TW * jj;
            if (r < rb && c < kbsz && (ib > kb || c <= r)) A[(i0 + r) * n + k0 + c] = acc[i][jj];
          }
        __syncthreads();
      }
    }
  }

  if (INV) {
    // X = C^{-1} block column by block column, X^H kept in the upper triangle of A
    for (int j = 0; j < nblk; ++j) {
      const int64_t j0 = (int64_t)j * CB;
      const int jb = (int)(CB < (n - j0) ? (int64_t)CB : (n - j0));
      const int gend = min(nblk, (j / inv_group + 1) * inv_group);
      for (int ib = j + 1; ib < gend; ++ib) {
        const int64_t i0 = (int64_t)ib * CB;
        const int rb = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
        double2 acc[4][4];
        zero_acc(acc);
        for (int kb = j; kb < ib; ++kb) {
          const int64_t k0 = (int64_t)kb * CB;
          const int kbsz = (int)(CB < (n - k0) ? (int64_t)CB : (n - k0));
          load_blk(S2, A, n, i0, k0, rb, kbsz);  // C_ik (strictly lower block)
          if (kb == j)
            load_blk_adjU(S0, A, n, j0, jb);  // X_jj
          else
            load_blk_adj(S0, A, n, j0, k0, jb, kbsz);  // X_kj = (A_jk)^H
          __syncthreads();
          mma_tile<false>(S2, S0, kbsz, acc);
          __syncthreads();
        }
        // X_ij = -C_ii^{-1} acc
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) S2[(ty + TW * i) * PITCH + tx + TW * jj] = acc[i][jj];
        load_blk_adjU(S0, A, n, i0, rb);  // C_ii^{-1}
        __syncthreads();
        zero_acc(acc);
        mma_tile<false>(S0, S2, rb, acc);
        __syncthreads();
        // A[j0 + c][i0 + r] = conj(X_ij[r][c]) = -conj(acc[r][c])
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const int r = ty + TW * i, c = tx + TW * jj;
            if (r < rb && c < jb) A[(j0 + c) * n + i0 + r] = make_double2(-acc[i][jj].x, acc[i][jj].y);
          }
        __syncthreads();
      }
    }
  }

  // reductions
  for (int w = CT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s_red[0][threadIdx.x] += s_red[0][threadIdx.x + w];
      s_red[1][threadIdx.x] += s_red[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *logdet = 2.0 * s_ld;
    *trace = make_double2(s_red[0][0], s_red[1][0]);
    *info = s_bad;
  }
}

template <bool INV>
__global__ void __launch_bounds__(CT, 4) k_chol_inv(const float2* __restrict__ Mall,
                                                    double2* __restrict__ Aall,
                                                    double* __restrict__ logdet,
                                                    double2* __restrict__ trace,
                                                    int* __restrict__ info, int64_t n,
                                                    int inv_group) {
  const int64_t p = blockIdx.x;
  chol_inv_problem<INV>(Mall + p * n * n, Aall + p * n * n, logdet + p, trace + p, info + p, n,
                        inv_group);
}

// Problems of different sizes in one launch (one CTA each).
__global__ void __launch_bounds__(CT, 4) k_chol_inv_grouped(const CholProblem* __restrict__ probs,
                                                            double* __restrict__ logdet,
                                                            double2* __restrict__ trace,
                                                            int* __restrict__ info) {
  const CholProblem pr = probs[blockIdx.x];
  chol_inv_problem<true>(pr.M, pr.A, logdet + blockIdx.x, trace + blockIdx.x, info + blockIdx.x,
                         pr.n, 1 << 30);
}

// grouped A = I - M (lower) and Z = X^H - I, blockIdx.y = problem
__global__ void k_chol_prep_grouped(const CholProblem* __restrict__ probs) {
  const CholProblem pr = probs[blockIdx.y];
  const int64_t n = pr.n, total = n * n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / n, c = e % n;
    if (c <= r) {
      const float2 m = pr.M[e];
      pr.A[e] = make_double2((r == c ? 1.0 : 0.0) - (double)m.x, -(double)m.y);
    }
  }
}

__global__ void k_chol_final_grouped(const CholProblem* __restrict__ probs) {
  const CholProblem pr = probs[blockIdx.y];
  const int64_t n = pr.n, total = n * n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / n, c = e % n;
    float2 z = make_float2(0.f, 0.f);
    if (c >= r) {
      const double2 a = pr.A[e];
      z = make_float2((float)(a.x - (r == c ? 1.0 : 0.0)), (float)a.y);
    }
    pr.Z[e] = z;
  }
}

// A = I - M on the lower triangle of every problem (FP64)
__global__ void k_chol_prep(const float2* __restrict__ M, double2* __restrict__ A, int64_t n,
                            int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i % (n * n), r = e / n, c = e % n;
    if (c <= r) {
      const float2 m = M[i];
      A[i] = make_double2((r == c ? 1.0 : 0.0) - (double)m.x, -(double)m.y);
    }
  }
}

// Z = X^H - I from the upper triangle of A (complex64), zero below the diagonal
__global__ void k_chol_final(const double2* __restrict__ A, float2* __restrict__ Z, int64_t n,
                             int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i % (n * n), r = e / n, c = e % n;
    float2 z = make_float2(0.f, 0.f);
    if (c >= r) {
      const double2 a = A[i];
      z = make_float2((float)(a.x - (r == c ? 1.0 : 0.0)), (float)a.y);
    }
    Z[i] = z;
  }
}

// Operands of the tensor-core inverse levels from A (C in the lower triangle, U = C^{-H} in
// the upper triangle of each kInvGroup diagonal group):
//   Z  = U - I inside the diagonal groups' upper triangles, 0 below the diagonal (the levels
//        write the upper off-group blocks);
//   Zl = U^H - I = C^{-1} - I inside the diagonal groups' lower triangles, 0 elsewhere (the
//        levels write the lower off-group blocks they need later);
//   Zc = -C on the strictly lower off-group blocks (other entries are not written).
// 32 x 32 tiles; the transposed reads of Zl go through shared memory.
__global__ void __launch_bounds__(256) k_chol_split(const double2* __restrict__ Aall,
                                                   float2* __restrict__ Zall,
                                                   float2* __restrict__ Zlall,
                                                   float2* __restrict__ Zcall, int64_t n) {
  __shared__ double2 tile[32][33];
  const int64_t p = blockIdx.z;
  const double2* A = Aall + p * n * n;
  float2* Z = Zall + p * n * n;
  float2* Zl = Zlall + p * n * n;
  float2* Zc = Zcall + p * n * n;
  const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
  const bool same_group = (i0 / kInvGroup) == (j0 / kInvGroup);
  const bool mirror = same_group && i0 >= j0;  // lower tile of a group: needs U^H
  if (mirror) {
    for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
      const int64_t r = j0 + ty, c = i0 + threadIdx.x;  // upper tile (j0, i0)
      tile[ty][threadIdx.x] = (r < n && c < n && c >= r) ? A[r * n + c] : make_double2(0, 0);
    }
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    const int64_t i = i0 + ty, j = j0 + threadIdx.x;
    if (i >= n || j >= n) continue;
    const int64_t e = i * n + j;
    const float d = (i == j) ? 1.f : 0.f;
    if (j >= i) {
      if (same_group) {
        const double2 a = A[e];
        Z[e] = make_float2((float)(a.x - d), (float)a.y);
      }
    } else {
      Z[e] = make_float2(0.f, 0.f);
      if (!same_group) {
        const double2 a = A[e];
        Zc[e] = make_float2((float)(-a.x), (float)(-a.y));
      }
    }
    if (i >= j) {
      if (mirror) {
        const double2 u = tile[threadIdx.x][ty];  // A[j][i] = U[j][i]
        Zl[e] = make_float2((float)(u.x - d), (float)(-u.y));
      } else {
        Zl[e] = make_float2(0.f, 0.f);
      }
    } else {
      Zl[e] = make_float2(0.f, 0.f);
    }
  }
}

// Zl[r1 + c][r0 + r] = conj(Z[r0 + r][r1 + c]) for r < b, c < b1 (a level's result, kept as
// the lower-triangle operand of the next level)
__global__ void k_block_adjoint(const float2* __restrict__ Zall, float2* __restrict__ Zlall,
                                int64_t n, int64_t r0, int64_t r1, int64_t b, int64_t b1) {
  __shared__ float2 tile[32][33];
  const int64_t p = blockIdx.z;
  const float2* Z = Zall + p * n * n;
  float2* Zl = Zlall + p * n * n;
  const int64_t rt = (int64_t)blockIdx.y * 32, ct = (int64_t)blockIdx.x * 32;
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    const int64_t r = rt + ty, c = ct + threadIdx.x;
    tile[ty][threadIdx.x] = (r < b && c < b1) ? Z[(r0 + r) * n + r1 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    const int64_t c = ct + ty, r = rt + threadIdx.x;  // output row r1 + c, column r0 + r
    if (r < b && c < b1) {
      const float2 v = tile[threadIdx.x][ty];
      Zl[(r1 + c) * n + r0 + r] = make_float2(v.x, -v.y);
    }
  }
}

}  // namespace

void launch_chol_inv(const float2* M, double2* A, float2* Z, double* logdet, double2* trace,
                     int* info, int64_t Np, int64_t nprob, cudaStream_t s) {
  const size_t smem = (size_t)3 * CB * PITCH * sizeof(double2);
  const int64_t total = Np * Np * nprob;
  k_chol_prep<<<grid_for(total, 256), 256, 0, s>>>(M, A, Np, total);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  if (Z) {
    static bool set = false;
    if (!set) {
      CQ_CHECK_CUDA(cudaFuncSetAttribute(k_chol_inv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
      set = true;
    }
    k_chol_inv<true><<<(unsigned)nprob, CT, smem, s>>>(M, A, logdet, trace, info, Np, 1 << 30);
    count_launch();
    CQ_CHECK_CUDA(cudaGetLastError());
    k_chol_final<<<grid_for(total, 256), 256, 0, s>>>(A, Z, Np, total);
  } else {
    static bool set = false;
    if (!set) {
      CQ_CHECK_CUDA(cudaFuncSetAttribute(k_chol_inv<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      set = true;
    }
    k_chol_inv<false><<<(unsigned)nprob, CT, smem, s>>>(M, A, logdet, trace, info, Np, 1 << 30);
  }
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void launch_chol_group_inv(const float2* M, double2* A, double* logdet, double2* trace, int* info,
                           int64_t Np, int64_t nprob, cudaStream_t s) {
  const size_t smem = (size_t)3 * CB * PITCH * sizeof(double2);
  const int64_t total = Np * Np * nprob;
  k_chol_prep<<<grid_for(total, 256), 256, 0, s>>>(M, A, Np, total);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  static bool set = false;
  if (!set) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(k_chol_inv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    set = true;
  }
  k_chol_inv<true><<<(unsigned)nprob, CT, smem, s>>>(M, A, logdet, trace, info, Np, kInvGroup / CB);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void launch_chol_split(const double2* A, float2* Z, float2* Zl, float2* Zc, int64_t Np,
                       int64_t nprob, cudaStream_t s) {
  CQ_REQUIRE(nprob <= 65535, COQUI_B200_EINVAL, "chol_split: too many problems per launch");
  const unsigned nt = (unsigned)((Np + 31) / 32);
  k_chol_split<<<dim3(nt, nt, (unsigned)nprob), dim3(32, 8), 0, s>>>(A, Z, Zl, Zc, Np);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void launch_block_adjoint(const float2* Z, float2* Zl, int64_t Np, int64_t r0, int64_t r1,
                          int64_t b, int64_t b1, int64_t nprob, cudaStream_t s) {
  CQ_REQUIRE(nprob <= 65535 && r0 + b <= r1 && r1 + b1 <= Np, COQUI_B200_EINVAL,
             "block_adjoint: bad block");
  const dim3 g((unsigned)((b1 + 31) / 32), (unsigned)((b + 31) / 32), (unsigned)nprob);
  k_block_adjoint<<<g, dim3(32, 8), 0, s>>>(Z, Zl, Np, r0, r1, b, b1);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void launch_chol_inv_grouped(const std::vector<CholProblem>& probs, DevBuf<unsigned char>& table,
                             double* logdet, double2* trace, int* info, cudaStream_t s) {
  if (probs.empty()) return;
  const int64_t np = (int64_t)probs.size();
  CQ_REQUIRE(np <= 65535, COQUI_B200_EINVAL, "chol grouped: at most 65535 problems per launch");
  table.ensure(np * sizeof(CholProblem));
  CQ_CHECK_CUDA(cudaMemcpyAsync(table.p, probs.data(), np * sizeof(CholProblem),
                                cudaMemcpyHostToDevice, s));
  const CholProblem* t = (const CholProblem*)table.p;
  int64_t nmax = 0;
  for (const auto& p : probs) nmax = std::max(nmax, p.n);
  const unsigned gx = (unsigned)std::min<int64_t>((nmax * nmax + 255) / 256, 1024);
  k_chol_prep_grouped<<<dim3(gx, (unsigned)np), 256, 0, s>>>(t);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  const size_t smem = (size_t)3 * CB * PITCH * sizeof(double2);
  static bool set = false;
  if (!set) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(k_chol_inv_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    set = true;
  }
  k_chol_inv_grouped<<<(unsigned)np, CT, smem, s>>>(t, logdet, trace, info);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  k_chol_final_grouped<<<dim3(gx, (unsigned)np), 256, 0, s>>>(t);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

}  // namespace cq
