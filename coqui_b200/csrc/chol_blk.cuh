// Blocked FP64 Cholesky / log-determinant / triangular inverse of one problem per CTA.
// Included once per block size inside a namespace that defines
//   CB (block edge), CT (threads), PITCH (shared-memory row pitch in double2, CB + 1), MINB
//   (CTAs per SM for the launch bounds), DMMA (block products on the FP64 tensor cores; needs
//   CB = 32 and CT = 64), AR x AC (a thread's accumulator tile: 2 x 8 for DMMA, else RT x CTT
//   with the thread grid TWR = CB / RT by TWC = CB / CTT, CT = TWR * TWC)
// and the complex helpers cmul_, cmulc_, conj_.  (No include guard: it is meant to be
// included more than once.)
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
// element (r, c) of I - M (M complex64, n x n row-major) in FP64
__device__ __forceinline__ double2 i_minus_m(const float2* M, int64_t n, int64_t r, int64_t c) {
  const float2 m = M[r * n + c];
  return make_double2((r == c ? 1.0 : 0.0) - (double)m.x, -(double)m.y);
}
// smem tile <- block of I - M (the first block column's reads: A = I - M is not stored)
__device__ __forceinline__ void load_blk_im(double2* S, const float2* M, int64_t n, int64_t r0,
                                            int64_t c0, int rb, int cb) {
  double2 v[CB * CB / CT];
#pragma unroll
  for (int u = 0; u < CB * CB / CT; ++u) {
    const int i = threadIdx.x + u * CT;
    const int r = i / CB, c = i % CB;
    v[u] = (r < rb && c < cb) ? i_minus_m(M, n, r0 + r, c0 + c) : make_double2(0, 0);
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

// Register tile of a 32 x 32 block product: acc[i][j] is the element (acc_row(i, j),
// acc_col(i, j)).  FMA form: thread (ty, tx) of the TWR x TWC grid holds rows ty + TWR i and
// columns tx + TWC j.  DMMA form (FP64 tensor-core mma.sync m8n8k4, DMMA = true, two warps):
// warp w holds the 8 x 8 tiles of tile rows 2w, 2w + 1 and all four tile columns; lane l
// holds elements (8 (2w + i) + l / 4, 8 (j / 2) + 2 (l % 4) + j % 2) of the accumulator
// fragments.
__device__ __forceinline__ int acc_row(int i, int j) {
  if constexpr (DMMA) return 8 * (2 * (int)(threadIdx.x >> 5) + i) + (int)((threadIdx.x & 31) >> 2);
  else return (int)(threadIdx.x / TWC) + TWR * i;
}
__device__ __forceinline__ int acc_col(int i, int j) {
  if constexpr (DMMA) return 8 * (j >> 1) + 2 * (int)(threadIdx.x & 3) + (j & 1);
  else return (int)(threadIdx.x % TWC) + TWC * j;
}

// D (8 x 8, two values per lane) += A (8 x 4, one per lane) * B (4 x 8, one per lane), FP64.
// Not volatile: the compiler may interleave independent products (their operands and
// accumulators are the only dependencies).
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// acc += sign * sum_k X[r][k] * Y'(k, c) over k < K, with Y'(k, c) = conj(Y[c][k]) if ADJ_Y
// (product with Y^H) else Y[k][c]; sign = -1 if SUB.  The DMMA form runs K up to a multiple of
// four: the staging tiles hold zeros beyond their valid extent.
template <bool ADJ_Y, bool SUB>
__device__ __forceinline__ void block_mma(const double2* X, const double2* Y, int K,
                                          double2 (&acc)[AR][AC]) {
  if constexpr (DMMA) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, g = l >> 2, q = l & 3;
    const double sg = SUB ? -1.0 : 1.0;
    for (int k0 = 0; k0 < K; k0 += 4) {
      const int k = k0 + q;
      double2 x[AR], y[4];
#pragma unroll
      for (int i = 0; i < AR; ++i) x[i] = X[(8 * (2 * w + i) + g) * PITCH + k];
#pragma unroll
      for (int t = 0; t < 4; ++t) y[t] = ADJ_Y ? Y[(8 * t + g) * PITCH + k] : Y[k * PITCH + 8 * t + g];
      // four passes over the AR x 4 fragment pairs: consecutive products feed different
      // accumulators, and every accumulator still receives its terms in the same order
      // (real part: xr yr then the xi yi term; imaginary part: the xi yr term then xr yi)
      double xr[AR], xi[AR];
#pragma unroll
      for (int i = 0; i < AR; ++i) {
        xr[i] = sg * x[i].x;
        xi[i] = sg * x[i].y;
      }
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int t = 0; t < 4; ++t) dmma(acc[i][2 * t].x, acc[i][2 * t + 1].x, xr[i], y[t].x);
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int t = 0; t < 4; ++t)  // x conj(y): + xi yi; x y: - xi yi
          dmma(acc[i][2 * t].x, acc[i][2 * t + 1].x, ADJ_Y ? xi[i] : -xi[i], y[t].y);
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int t = 0; t < 4; ++t)  // x conj(y): + xi yr (then - xr yi); x y: + xr yi (then + xi yr)
          dmma(acc[i][2 * t].y, acc[i][2 * t + 1].y, ADJ_Y ? xi[i] : xr[i], ADJ_Y ? y[t].x : y[t].y);
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int t = 0; t < 4; ++t)
          dmma(acc[i][2 * t].y, acc[i][2 * t + 1].y, ADJ_Y ? -xr[i] : xi[i], ADJ_Y ? y[t].y : y[t].x);
    }
  } else {
    const int tx = threadIdx.x % TWC, ty = threadIdx.x / TWC;
    for (int k = 0; k < K; ++k) {
      double2 a[AR], b[AC];
#pragma unroll
      for (int i = 0; i < AR; ++i) {
        a[i] = X[(ty + TWR * i) * PITCH + k];
        if (SUB) a[i] = make_double2(-a[i].x, -a[i].y);
      }
#pragma unroll
      for (int j = 0; j < AC; ++j)
        b[j] = ADJ_Y ? conj_(Y[(tx + TWC * j) * PITCH + k]) : Y[k * PITCH + tx + TWC * j];
#pragma unroll
      for (int i = 0; i < AR; ++i)  // four passes of AR * AC independent FMAs (no back-to-back
#pragma unroll                   // dependency inside a complex multiply-add)
        for (int j = 0; j < AC; ++j) acc[i][j].x = fma(-a[i].y, b[j].y, acc[i][j].x);
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int j = 0; j < AC; ++j) acc[i][j].y = fma(a[i].y, b[j].x, acc[i][j].y);
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int j = 0; j < AC; ++j) acc[i][j].x = fma(a[i].x, b[j].x, acc[i][j].x);
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int j = 0; j < AC; ++j) acc[i][j].y = fma(a[i].x, b[j].y, acc[i][j].y);
    }
  }
}

template <bool ADJ_Y>
__device__ __forceinline__ void mma_tile(const double2* X, const double2* Y, int K,
                                         double2 (&acc)[AR][AC]) {
  block_mma<ADJ_Y, false>(X, Y, K, acc);
}

// acc -= sum_k X[r][k] conj(Y[c][k])  (A - X Y^H)
__device__ __forceinline__ void mma_tile_sub(const double2* X, const double2* Y, int K,
                                             double2 (&acc)[AR][AC]) {
  block_mma<true, true>(X, Y, K, acc);
}

__device__ __forceinline__ void zero_acc(double2 (&acc)[AR][AC]) {
#pragma unroll
  for (int i = 0; i < AR; ++i)
#pragma unroll
    for (int j = 0; j < AC; ++j) acc[i][j] = make_double2(0, 0);
}

// acc <- block (i0.., k0..) of A, or of I - M (from_m, the first block column), restricted
// to rb x kbsz and, unless off_diag, to the lower triangle; the source is chosen once for the
// whole tile so that all its loads are issued back to back
__device__ __forceinline__ void acc_init(double2 (&acc)[AR][AC], const double2* A, const float2* M,
                                         bool from_m, int64_t n, int64_t i0, int64_t k0, int rb,
                                         int kbsz, bool off_diag) {
  if (from_m) {
#pragma unroll
    for (int i = 0; i < AR; ++i)
#pragma unroll
      for (int jj = 0; jj < AC; ++jj) {
        const int r = acc_row(i, jj), c = acc_col(i, jj);
        acc[i][jj] = (r < rb && c < kbsz && (off_diag || c <= r)) ? i_minus_m(M, n, i0 + r, k0 + c)
                                                                  : make_double2(0, 0);
      }
  } else {
#pragma unroll
    for (int i = 0; i < AR; ++i)
#pragma unroll
      for (int jj = 0; jj < AC; ++jj) {
        const int r = acc_row(i, jj), c = acc_col(i, jj);
        acc[i][jj] = (r < rb && c < kbsz && (off_diag || c <= r)) ? A[(i0 + r) * n + k0 + c]
                                                                  : make_double2(0, 0);
      }
  }
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
// per group of CT / CB lanes of a warp (partial dot products reduced by shuffles).
__device__ void invert_lower(const double2* S, double2* Sinv, int n) {
  constexpr int LPC = CT / CB;  // lanes per column
  for (int i = threadIdx.x; i < CB * CB; i += CT) Sinv[(i / CB) * PITCH + i % CB] = make_double2(0, 0);
  __syncthreads();
  const int c = threadIdx.x / LPC, sub = threadIdx.x % LPC;
  const bool col = c < n;
  if (col && sub == 0) Sinv[c * PITCH + c] = make_double2(1.0 / S[c * PITCH + c].x, 0.0);
  __syncwarp();
  for (int r = 1; r < n; ++r) {
    double ax = 0, ay = 0;
    if (col && r > c)
      for (int k = c + sub; k < r; k += LPC) {
        const double2 u = cmul_(S[r * PITCH + k], Sinv[k * PITCH + c]);
        ax += u.x;
        ay += u.y;
      }
#pragma unroll
    for (int off = LPC / 2; off > 0; off >>= 1) {
      ax += __shfl_xor_sync(0xffffffffu, ax, off);
      ay += __shfl_xor_sync(0xffffffffu, ay, off);
    }
    if (col && r > c && sub == 0) {
      const double inv = -1.0 / S[r * PITCH + r].x;
      Sinv[r * PITCH + c] = make_double2(ax * inv, ay * inv);
    }
    __syncwarp();
  }
  __syncthreads();
}

// Column j of X = C^{-1} below the diagonal within its diagonal group (blocks j+1 .. gend-1):
//   X_ij = -C_ii^{-1} sum_{k=j}^{i-1} C_ik X_kj,
// with C_ik in the lower triangle of A, C_ii^{-H} in the upper triangle of the diagonal
// blocks; X_ij is kept as its adjoint in the upper block (j, i).  Columns are independent.
__device__ void inverse_column(double2* A, int64_t n, int j, int gend, double2* S0, double2* S1) {
  const int64_t j0 = (int64_t)j * CB;
  const int jb = (int)(CB < (n - j0) ? (int64_t)CB : (n - j0));
  for (int ib = j + 1; ib < gend; ++ib) {
    const int64_t i0 = (int64_t)ib * CB;
    const int rb = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
    double2 acc[AR][AC];
    zero_acc(acc);
    for (int kb = j; kb < ib; ++kb) {
      const int64_t k0 = (int64_t)kb * CB;
      const int kbsz = (int)(CB < (n - k0) ? (int64_t)CB : (n - k0));
      load_blk(S1, A, n, i0, k0, rb, kbsz);  // C_ik (strictly lower block)
      if (kb == j)
        load_blk_adjU(S0, A, n, j0, jb);  // X_jj
      else
        load_blk_adj(S0, A, n, j0, k0, jb, kbsz);  // X_kj = (A_jk)^H
      __syncthreads();
      mma_tile<false>(S1, S0, kbsz, acc);
      __syncthreads();
    }
    // X_ij = -C_ii^{-1} acc
#pragma unroll
    for (int i = 0; i < AR; ++i)
#pragma unroll
      for (int jj = 0; jj < AC; ++jj) S1[acc_row(i, jj) * PITCH + acc_col(i, jj)] = acc[i][jj];
    load_blk_adjU(S0, A, n, i0, rb);  // C_ii^{-1}
    __syncthreads();
    zero_acc(acc);
    mma_tile<false>(S0, S1, rb, acc);
    __syncthreads();
    // A[j0 + c][i0 + r] = conj(X_ij[r][c]) = -conj(acc[r][c])
#pragma unroll
    for (int i = 0; i < AR; ++i)
#pragma unroll
      for (int jj = 0; jj < AC; ++jj) {
        const int r = acc_row(i, jj), c = acc_col(i, jj);
        if (r < rb && c < jb) A[(j0 + c) * n + i0 + r] = make_double2(-acc[i][jj].x, acc[i][jj].y);
      }
    __syncthreads();
  }
}

// ---- tiled factorisation: one problem spread over many CTAs, one launch per phase of each
// block column j (diagonal block; panel blocks; trailing blocks), then the group inverse ----

// diagonal block j: factor and invert in shared memory, C_jj^{-H} into the upper triangle,
// ln det contribution added to *logdet, *info set for a non-positive pivot
__device__ void tiled_diag(const float2* M, double2* A, int64_t n, int j, double* logdet,
                           int* info) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* S0 = reinterpret_cast<double2*>(smem_raw);
  double2* S1 = S0 + CB * PITCH;
  __shared__ double s_ld;
  __shared__ int s_bad;
  if (threadIdx.x == 0) {
    s_ld = 0.0;
    s_bad = 0;
  }
  const int64_t j0 = (int64_t)j * CB;
  const int jb = (int)(CB < (n - j0) ? (int64_t)CB : (n - j0));
  if (j == 0)
    load_blk_im(S0, M, n, j0, j0, jb, jb);
  else
    load_blk(S0, A, n, j0, j0, jb, jb);
  __syncthreads();
  factor_diag(S0, jb, &s_ld, &s_bad);
  invert_lower(S0, S1, jb);
  store_blk_adjU(S1, A, n, j0, jb);
  if (threadIdx.x == 0) {
    *logdet += 2.0 * s_ld;
    if (s_bad) *info = 1;
  }
}

// panel block (i, j), i > j: L_ij = A_ij C_jj^{-H}
__device__ void tiled_panel(const float2* M, double2* A, int64_t n, int j, int ib) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* S0 = reinterpret_cast<double2*>(smem_raw);
  double2* S1 = S0 + CB * PITCH;
  const int64_t j0 = (int64_t)j * CB, i0 = (int64_t)ib * CB;
  const int jb = (int)(CB < (n - j0) ? (int64_t)CB : (n - j0));
  const int rb = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
  if (j == 0)
    load_blk_im(S0, M, n, i0, j0, rb, jb);
  else
    load_blk(S0, A, n, i0, j0, rb, jb);
  load_blk_adjU(S1, A, n, j0, jb);  // C_jj^{-1}
  __syncthreads();
  double2 acc[AR][AC];
  zero_acc(acc);
  mma_tile<true>(S0, S1, jb, acc);
#pragma unroll
  for (int i = 0; i < AR; ++i)
#pragma unroll
    for (int jj = 0; jj < AC; ++jj) {
      const int r = acc_row(i, jj), c = acc_col(i, jj);
      if (r < rb && c < jb) A[(i0 + r) * n + j0 + c] = acc[i][jj];
    }
}

// Trailing update of block (ib, kb) by the block columns j .. j + cols - 1 (lower triangle
// only when ib == kb): A_ik -= sum_c L_ic L_kc^H, the rank-CB products one column at a time,
// with the block held in FP64 registers in between rather than stored and reloaded, so the
// block is read and written once for all of them.
__device__ void tiled_update_cols(const float2* M, double2* A, int64_t n, int j, int cols, int ib,
                                  int kb) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* S0 = reinterpret_cast<double2*>(smem_raw);
  double2* S1 = S0 + CB * PITCH;
  const int64_t i0 = (int64_t)ib * CB, k0 = (int64_t)kb * CB;
  const int rb = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
  const int kbsz = (int)(CB < (n - k0) ? (int64_t)CB : (n - k0));
  double2 acc[AR][AC];
  acc_init(acc, A, M, j == 0, n, i0, k0, rb, kbsz, ib > kb);
  for (int c = 0; c < cols; ++c) {
    const int64_t jc = (int64_t)(j + c) * CB;
    const int jb = (int)(CB < (n - jc) ? (int64_t)CB : (n - jc));
    if (c > 0) __syncthreads();  // every warp is done with the previous column's blocks
    load_blk(S0, A, n, i0, jc, rb, jb);
    load_blk(S1, A, n, k0, jc, kbsz, jb);
    __syncthreads();
    mma_tile_sub(S0, S1, jb, acc);
  }
#pragma unroll
  for (int i = 0; i < AR; ++i)
#pragma unroll
    for (int jj = 0; jj < AC; ++jj) {
      const int r = acc_row(i, jj), c = acc_col(i, jj);
      if (r < rb && c < kbsz && (ib > kb || c <= r)) A[(i0 + r) * n + k0 + c] = acc[i][jj];
    }
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
  // two staging blocks: the diagonal block and its inverse, then (panel) a panel block and the
  // inverse, (trailing update) the two panel blocks, (inverse) C_ik and X_kj
  double2* S0 = reinterpret_cast<double2*>(smem_raw);
  double2* S1 = S0 + CB * PITCH;
  __shared__ double s_ld;
  __shared__ int s_bad;
  __shared__ double s_red[2][CT];
  const int nblk = (int)((n + CB - 1) / CB);

  if (threadIdx.x == 0) {
    s_ld = 0.0;
    s_bad = 0;
  }
  // trace of M; A = I - M is read from M in block column 0 (every lower block of A is written
  // there: the panel and the trailing update of column 0)
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
    if (j == 0)
      load_blk_im(S0, M, n, j0, j0, jb, jb);
    else
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
      if (j == 0)
        load_blk_im(S0, M, n, i0, j0, rb, jb);
      else
        load_blk(S0, A, n, i0, j0, rb, jb);
      __syncthreads();
      double2 acc[AR][AC];
      zero_acc(acc);
      mma_tile<true>(S0, S1, jb, acc);
      __syncthreads();
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int jj = 0; jj < AC; ++jj) {
          const int r = acc_row(i, jj), c = acc_col(i, jj);
          if (r < rb && c < jb) A[(i0 + r) * n + j0 + c] = acc[i][jj];
        }
      __syncthreads();
    }
    // 3. trailing update of the lower triangle: A_ik -= L_ij L_kj^H
    for (int kb = j + 1; kb < nblk; ++kb) {
      const int64_t k0 = (int64_t)kb * CB;
      const int kbsz = (int)(CB < (n - k0) ? (int64_t)CB : (n - k0));
      load_blk(S1, A, n, k0, j0, kbsz, jb);
      for (int ib = kb; ib < nblk; ++ib) {
        const int64_t i0 = (int64_t)ib * CB;
        const int rb = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
        load_blk(S0, A, n, i0, j0, rb, jb);
        __syncthreads();
        double2 acc[AR][AC];
        acc_init(acc, A, M, j == 0, n, i0, k0, rb, kbsz, ib > kb);  // loads in flight early
        mma_tile_sub(S0, S1, jb, acc);
#pragma unroll
        for (int i = 0; i < AR; ++i)
#pragma unroll
          for (int jj = 0; jj < AC; ++jj) {
            const int r = acc_row(i, jj), c = acc_col(i, jj);
            if (r < rb && c < kbsz && (ib > kb || c <= r)) A[(i0 + r) * n + k0 + c] = acc[i][jj];
          }
        __syncthreads();
      }
    }
  }

  if (INV) {
    // X = C^{-1} block column by block column, X^H kept in the upper triangle of A
    for (int j = 0; j < nblk; ++j)
      inverse_column(A, n, j, min(nblk, (j / inv_group + 1) * inv_group), S0, S1);
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

// The same factorisation in left-looking (Crout) order: block column j is formed from I - M
// and the finished columns kb < j, A_ij - sum_kb L_ib,kb L_j,kb^H, so each block of M is read
// once and each block of C written once (the right-looking order above reads and rewrites the
// trailing lower triangle after every column).  Both staging blocks hold the two panel blocks
// of a product; C_jj^{-1} is reloaded from the upper triangle of the diagonal block, where
// C_jj^{-H} is kept.  Every block starts from I - M and has the same block products
// subtracted in the same order (kb = 0, 1, ...) in FP64 as in the right-looking order, which
// keeps the running sums in global memory: the results are identical.
template <bool INV>
__device__ __forceinline__ void chol_inv_problem_left(const float2* __restrict__ M,
                                                      double2* __restrict__ A,
                                                      double* __restrict__ logdet,
                                                      double2* __restrict__ trace,
                                                      int* __restrict__ info, int64_t n,
                                                      int inv_group) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* S0 = reinterpret_cast<double2*>(smem_raw);
  double2* S1 = S0 + CB * PITCH;
  __shared__ double s_ld;
  __shared__ int s_bad;
  __shared__ double s_red[2][CT];
  const int nblk = (int)((n + CB - 1) / CB);

  if (threadIdx.x == 0) {
    s_ld = 0.0;
    s_bad = 0;
  }
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
    // 1. diagonal block: (I - M)_jj - sum_kb L_j,kb L_j,kb^H, factor, invert
    double2 acc[AR][AC];
    acc_init(acc, A, M, true, n, j0, j0, jb, jb, false);
    for (int kb = 0; kb < j; ++kb) {  // blocks kb < j are full
      load_blk(S0, A, n, j0, (int64_t)kb * CB, jb, CB);
      __syncthreads();
      mma_tile_sub(S0, S0, CB, acc);
      __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < AR; ++i)
#pragma unroll
      for (int jj = 0; jj < AC; ++jj) S0[acc_row(i, jj) * PITCH + acc_col(i, jj)] = acc[i][jj];
    __syncthreads();
    factor_diag(S0, jb, &s_ld, &s_bad);
    invert_lower(S0, S1, jb);
    store_blk_adjU(S1, A, n, j0, jb);  // C_jj^{-H} in the upper triangle
    __syncthreads();
    // 2. panel: L_ib,j = [(I - M)_ib,j - sum_kb L_ib,kb L_j,kb^H] C_jj^{-H}
    for (int ib = j + 1; ib < nblk; ++ib) {
      const int64_t i0 = (int64_t)ib * CB;
      const int rb = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
      acc_init(acc, A, M, true, n, i0, j0, rb, jb, true);
      for (int kb = 0; kb < j; ++kb) {
        const int64_t k0 = (int64_t)kb * CB;
        load_blk(S0, A, n, i0, k0, rb, CB);
        load_blk(S1, A, n, j0, k0, jb, CB);
        __syncthreads();
        mma_tile_sub(S0, S1, CB, acc);
        __syncthreads();
      }
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int jj = 0; jj < AC; ++jj) S0[acc_row(i, jj) * PITCH + acc_col(i, jj)] = acc[i][jj];
      load_blk_adjU(S1, A, n, j0, jb);  // C_jj^{-1}
      __syncthreads();
      double2 l[AR][AC];
      zero_acc(l);
      mma_tile<true>(S0, S1, jb, l);
#pragma unroll
      for (int i = 0; i < AR; ++i)
#pragma unroll
        for (int jj = 0; jj < AC; ++jj) {
          const int r = acc_row(i, jj), c = acc_col(i, jj);
          if (r < rb && c < jb) A[(i0 + r) * n + j0 + c] = l[i][jj];
        }
      __syncthreads();
    }
  }

  if (INV) {
    for (int j = 0; j < nblk; ++j)
      inverse_column(A, n, j, min(nblk, (j / inv_group + 1) * inv_group), S0, S1);
  }

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
__global__ void __launch_bounds__(CT, MINB) k_chol_inv_left(const float2* __restrict__ Mall,
                                                         double2* __restrict__ Aall,
                                                         double* __restrict__ logdet,
                                                         double2* __restrict__ trace,
                                                         int* __restrict__ info, int64_t n,
                                                         int inv_group) {
  const int64_t p = blockIdx.x;
  chol_inv_problem_left<INV>(Mall + p * n * n, Aall + p * n * n, logdet + p, trace + p, info + p,
                             n, inv_group);
}

template <bool INV>
__global__ void __launch_bounds__(CT, MINB) k_chol_inv(const float2* __restrict__ Mall,
                                                    double2* __restrict__ Aall,
                                                    double* __restrict__ logdet,
                                                    double2* __restrict__ trace,
                                                    int* __restrict__ info, int64_t n,
                                                    int inv_group) {
  const int64_t p = blockIdx.x;
  chol_inv_problem<INV>(Mall + p * n * n, Aall + p * n * n, logdet + p, trace + p, info + p, n,
                        inv_group);
}

