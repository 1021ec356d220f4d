// Left-looking blocked FP64 Cholesky / log-determinant / group inverse of one problem per CTA,
// four warps, 32 x 32 blocks, two panel row blocks per step.
//
// Included once inside a namespace (chol.cu) that provides cmul_, cmulc_ and conj_.  The
// arithmetic of every element is that of the two-warp kernel in chol_blk.cuh (same products
// in the same order, same diagonal factorisation and inverse), so results are bit-identical;
// what differs is the data movement:
//  * the panel of block column j is formed two row blocks at a time (warps 0-1 on row block
//    i, warps 2-3 on row block i + 1), so each block L_j,k is read once per pair: 24 KB of
//    block loads per 32 x 32 x 32 product instead of 32 KB (an odd last row block is formed
//    by all four warps, one tile row each);
//  * blocks go from global to shared memory by cp.async (no staging registers), in K slices
//    of 32 / NS columns, optionally double-buffered (STAGES = 2) so the next slice's copies
//    are in flight during this one's products;
//  * shared blocks are stored unpadded with an XOR swizzle of 16-byte slots, element (r, c) at
//    r * 32 + (c ^ swz(r)): the DMMA operand reads (rows g, g + 1 of a fragment, four K
//    columns), row-wise copies and transposed stores all hit eight distinct slots per
//    quarter warp.
// Single-block products (the diagonal block's update, the inverse columns) spread the block's
// four 8-row tile rows over the four warps.

namespace p32 {

constexpr int CB = 32;
constexpr int NT = 128;  // four warps

__device__ __forceinline__ int swz(int r) { return ((r & 1) << 2) | ((r >> 1) & 3); }
// element (r, c) of a shared tile with rows of W values (W = 32: a whole block; W = 16: a
// half-width K slice of one)
template <int W = CB>
__device__ __forceinline__ int sidx(int r, int c) { return r * W + (c ^ swz(r)); }

// 16-byte global -> shared asynchronous copy; valid = false zero-fills (no bytes are read)
__device__ __forceinline__ void cp16(double2* dst, const double2* src, bool valid) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// S (32 rows of W) <- the tile (r0.., c0..) of the row-major ld x ld matrix G, zero outside
// rb x cb (async)
template <int W = CB>
__device__ __forceinline__ void cp_blk(double2* S, const double2* G, int64_t ld, int64_t r0,
                                       int64_t c0, int rb, int cb) {
#pragma unroll
  for (int u = 0; u < CB * W / NT; ++u) {
    const int i = threadIdx.x + u * NT, r = i / W, c = i % W;
    const bool v = r < rb && c < cb;
    cp16(S + sidx<W>(r, c), v ? G + (r0 + r) * ld + c0 + c : G, v);
  }
}

// S (lower triangle) <- adjoint of the upper triangle of the diagonal block at (r0, r0):
// S[c][r] = conj(G[r0 + r][r0 + c]) for c >= r, 0 elsewhere
__device__ __forceinline__ void load_adjU(double2* S, const double2* G, int64_t ld, int64_t r0,
                                          int nb) {
  double2 v[CB * CB / NT];
#pragma unroll
  for (int u = 0; u < CB * CB / NT; ++u) {
    const int i = threadIdx.x + u * NT, r = i / CB, c = i % CB;
    v[u] = (r < nb && c < nb && c >= r) ? conj_(G[(r0 + r) * ld + r0 + c]) : make_double2(0, 0);
  }
#pragma unroll
  for (int u = 0; u < CB * CB / NT; ++u) {
    const int i = threadIdx.x + u * NT;
    S[sidx(i % CB, i / CB)] = v[u];
  }
}

// S (lower triangle) <- the adjoint of a global block: S[c][r] = conj(G[r0 + r][c0 + c])
__device__ __forceinline__ void load_adj(double2* S, const double2* G, int64_t ld, int64_t r0,
                                         int64_t c0, int gr, int gc) {
  double2 v[CB * CB / NT];
#pragma unroll
  for (int u = 0; u < CB * CB / NT; ++u) {
    const int i = threadIdx.x + u * NT, r = i / CB, c = i % CB;
    v[u] = (r < gr && c < gc) ? conj_(G[(r0 + r) * ld + c0 + c]) : make_double2(0, 0);
  }
#pragma unroll
  for (int u = 0; u < CB * CB / NT; ++u) {
    const int i = threadIdx.x + u * NT;
    S[sidx(i % CB, i / CB)] = v[u];
  }
}

// upper triangle of the global diagonal block <- adjoint of the lower-triangular S
__device__ __forceinline__ void store_adjU(const double2* S, double2* G, int64_t ld, int64_t r0,
                                           int nb) {
#pragma unroll
  for (int u = 0; u < CB * CB / NT; ++u) {
    const int i = threadIdx.x + u * NT, r = i / CB, c = i % CB;
    if (r < nb && c < nb && r >= c) G[(r0 + c) * ld + r0 + r] = conj_(S[sidx(r, c)]);
  }
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// Register tile: a warp holds tile rows tr0 .. tr0 + AR - 1 (8 rows each) and all four tile
// columns; acc[i][j] is element (8 (tr0 + i) + lane / 4, 8 (j / 2) + 2 (lane % 4) + j % 2).
__device__ __forceinline__ int fr_row(int tr0, int i) { return 8 * (tr0 + i) + ((threadIdx.x & 31) >> 2); }
__device__ __forceinline__ int fr_col(int j) { return 8 * (j >> 1) + 2 * (threadIdx.x & 3) + (j & 1); }

// acc +/-= X Y' over k < K (K rounded up to a multiple of four; the tiles hold zeros beyond
// their valid extent), Y'(k, c) = conj(Y[c][k]) if ADJ_Y else Y[k][c]
// (tiles of row width W: X is 32 x W, Y is 32 x W if ADJ_Y, else 32 x 32 with K <= 32)
template <bool ADJ_Y, bool SUB, int AR, int W = CB>
__device__ __forceinline__ void mma_sw(const double2* X, const double2* Y, int K,
                                       double2 (&acc)[AR][8], int tr0) {
  const int l = threadIdx.x & 31, g = l >> 2, q = l & 3;
  const double sg = SUB ? -1.0 : 1.0;
  for (int k0 = 0; k0 < K; k0 += 4) {
    const int k = k0 + q;
    double2 x[AR], y[4];
#pragma unroll
    for (int i = 0; i < AR; ++i) x[i] = X[sidx<W>(8 * (tr0 + i) + g, k)];
#pragma unroll
    for (int t = 0; t < 4; ++t) y[t] = ADJ_Y ? Y[sidx<W>(8 * t + g, k)] : Y[sidx(k, 8 * t + g)];
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
      for (int t = 0; t < 4; ++t)
        dmma(acc[i][2 * t].x, acc[i][2 * t + 1].x, ADJ_Y ? xi[i] : -xi[i], y[t].y);
#pragma unroll
    for (int i = 0; i < AR; ++i)
#pragma unroll
      for (int t = 0; t < 4; ++t)
        dmma(acc[i][2 * t].y, acc[i][2 * t + 1].y, ADJ_Y ? xi[i] : xr[i], ADJ_Y ? y[t].x : y[t].y);
#pragma unroll
    for (int i = 0; i < AR; ++i)
#pragma unroll
      for (int t = 0; t < 4; ++t)
        dmma(acc[i][2 * t].y, acc[i][2 * t + 1].y, ADJ_Y ? -xr[i] : xi[i], ADJ_Y ? y[t].y : y[t].x);
  }
}

template <int AR>
__device__ __forceinline__ void zero(double2 (&acc)[AR][8]) {
#pragma unroll
  for (int i = 0; i < AR; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = make_double2(0, 0);
}

// acc <- block (i0.., k0..) of I - M, restricted to rb x kb and, unless off_diag, to the
// lower triangle
template <int AR, typename MT>
__device__ __forceinline__ void init_im(double2 (&acc)[AR][8], const MT* M, int64_t n,
                                        int64_t i0, int64_t k0, int rb, int kb, bool off_diag,
                                        int tr0) {
#pragma unroll
  for (int i = 0; i < AR; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int r = fr_row(tr0, i), c = fr_col(j);
      if (r < rb && c < kb && (off_diag || c <= r)) {
        const MT m = M[(i0 + r) * n + k0 + c];
        acc[i][j] = make_double2(((i0 + r) == (k0 + c) ? 1.0 : 0.0) - (double)m.x, -(double)m.y);
      } else {
        acc[i][j] = make_double2(0, 0);
      }
    }
}

template <int AR>
__device__ __forceinline__ void to_smem(double2* S, const double2 (&acc)[AR][8], int tr0) {
#pragma unroll
  for (int i = 0; i < AR; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) S[sidx(fr_row(tr0, i), fr_col(j))] = acc[i][j];
}

// In-place Cholesky of the lower triangle of S (n x n), sum ln C_ii added to *ld_acc by thread
// 0, *bad set for a non-positive pivot (the column step of chol_blk.cuh's factor_diag).
__device__ void factor_diag(double2* S, int n, double* ld_acc, int* bad) {
  double prev_inv = 1.0, prev_d = 1.0;
  for (int c = 0; c < n; ++c) {
    __syncthreads();
    double d = S[sidx(c, c)].x;
    const bool good = d > 0.0;
    d = good ? sqrt(d) : 1.0;
    const double inv = 1.0 / d;
    if (c > 0) {
      if (threadIdx.x == 0) S[sidx(c - 1, c - 1)] = make_double2(prev_d, 0.0);
      for (int r = c + threadIdx.x; r < n; r += NT) {
        double2& e = S[sidx(r, c - 1)];
        e.x *= prev_inv;
        e.y *= prev_inv;
      }
    }
    const int m = n - c - 1;
    const double inv2 = inv * inv;
    for (int idx = threadIdx.x; idx < m * m; idx += NT) {
      const int r = c + 1 + idx / m, s = c + 1 + idx % m;
      if (s <= r) {
        const double2 u = cmulc_(S[sidx(r, c)], S[sidx(s, c)]);
        double2& e = S[sidx(r, s)];
        e.x -= u.x * inv2;
        e.y -= u.y * inv2;
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
  if (threadIdx.x == 0) S[sidx(n - 1, n - 1)] = make_double2(prev_d, 0.0);
  __syncthreads();
}

// Sinv = inverse of the lower-triangular S (n x n): forward substitution, one column per lane
// pair (threads 0-63; the partial sums of a pair are combined by one shuffle, as in the
// two-warp kernel).
__device__ void invert_lower(const double2* S, double2* Sinv, int n) {
  for (int i = threadIdx.x; i < CB * CB; i += NT) Sinv[i] = make_double2(0, 0);
  __syncthreads();
  const int c = threadIdx.x >> 1, sub = threadIdx.x & 1;
  const bool col = c < n;
  if (col && sub == 0) Sinv[sidx(c, c)] = make_double2(1.0 / S[sidx(c, c)].x, 0.0);
  __syncwarp();
  for (int r = 1; r < n; ++r) {
    double ax = 0, ay = 0;
    if (col && r > c)
      for (int k = c + sub; k < r; k += 2) {
        const double2 u = cmul_(S[sidx(r, k)], Sinv[sidx(k, c)]);
        ax += u.x;
        ay += u.y;
      }
    ax += __shfl_xor_sync(0xffffffffu, ax, 1);
    ay += __shfl_xor_sync(0xffffffffu, ay, 1);
    if (col && r > c && sub == 0) {
      const double inv = -1.0 / S[sidx(r, r)].x;
      Sinv[sidx(r, c)] = make_double2(ax * inv, ay * inv);
    }
    __syncwarp();
  }
  __syncthreads();
}

// Column j of X = C^{-1} below the diagonal inside its group (blocks j+1 .. gend-1):
// X_ij = -C_ii^{-1} sum_{k=j}^{i-1} C_ik X_kj, kept as its adjoint in the upper block (j, i).
__device__ void inverse_column(double2* A, int64_t n, int j, int gend, double2* S0, double2* S1) {
  const int64_t j0 = (int64_t)j * CB;
  const int jb = (int)(CB < (n - j0) ? (int64_t)CB : (n - j0));
  const int w = threadIdx.x >> 5;
  for (int ib = j + 1; ib < gend; ++ib) {
    const int64_t i0 = (int64_t)ib * CB;
    const int rb = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
    double2 acc[1][8];
    zero(acc);
    for (int kb = j; kb < ib; ++kb) {
      const int64_t k0 = (int64_t)kb * CB;
      const int kbsz = (int)(CB < (n - k0) ? (int64_t)CB : (n - k0));
      cp_blk(S1, A, n, i0, k0, rb, kbsz);  // C_ik
      cp_commit();
      if (kb == j)
        load_adjU(S0, A, n, j0, jb);  // X_jj
      else
        load_adj(S0, A, n, j0, k0, jb, kbsz);  // X_kj = (A_jk)^H
      cp_wait<0>();
      __syncthreads();
      mma_sw<false, false, 1>(S1, S0, kbsz, acc, w);
      __syncthreads();
    }
    to_smem(S1, acc, w);
    load_adjU(S0, A, n, i0, rb);  // C_ii^{-1}
    __syncthreads();
    zero(acc);
    mma_sw<false, false, 1>(S0, S1, rb, acc, w);
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
      const int r = fr_row(w, 0), c = fr_col(jj);
      if (r < rb && c < jb) A[(j0 + c) * n + i0 + r] = make_double2(-acc[0][jj].x, acc[0][jj].y);
    }
    __syncthreads();
  }
}

// Runs compute(stage, it) for it = 0 .. nit - 1 on tiles that issue(stage, it) copies in
// (one commit group per call).  STAGES = 2: the copies of it + 1 are in flight while it is
// computed; STAGES = 1: copy, wait, compute.
template <int STAGES, typename Issue, typename Compute>
__device__ __forceinline__ void pipeline(int nit, Issue&& issue, Compute&& compute) {
  if (nit > 0) issue(0, 0);
  for (int it = 0; it < nit; ++it) {
    const int st = STAGES == 2 ? (it & 1) : 0;
    if (STAGES == 2 && it + 1 < nit) {
      issue(st ^ 1, it + 1);
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
    compute(st, it);
    __syncthreads();
    if (STAGES == 1 && it + 1 < nit) issue(0, it + 1);
  }
}

// Panel row blocks ib and, for AR = 2, ib + 1 of block column j (warps 0-1 on ib, warps 2-3
// on ib + 1, two tile rows each); AR = 1: row block ib alone, one tile row per warp.
// L_i,j = [(I - M)_i,j - sum_kb L_i,kb L_j,kb^H] C_jj^{-H} with C_jj^{-H} read from the upper
// triangle of the diagonal block.  SB / SA(stage, t): K-slice tiles; F(i): whole blocks.
template <int AR, int STAGES, int NS, typename MT, typename FB, typename FA, typename FF>
__device__ __forceinline__ void panel_step(const MT* __restrict__ M, double2* __restrict__ A,
                                           int64_t n, int j, int ib, FB&& SB, FA&& SA, FF&& F) {
  constexpr int W = CB / NS;
  const int w = threadIdx.x >> 5;
  const int team = AR == 2 ? (w >> 1) : 0;
  const int tr0 = AR == 2 ? 2 * (w & 1) : w;
  const int64_t j0 = (int64_t)j * CB, i0 = (int64_t)ib * CB, i1 = i0 + CB;
  const int jb = (int)(CB < (n - j0) ? (int64_t)CB : (n - j0));
  const int rb0 = (int)(CB < (n - i0) ? (int64_t)CB : (n - i0));
  const int rb1 = AR == 2 ? (int)(CB < (n - i1) ? (int64_t)CB : (n - i1)) : 0;
  const int64_t mi0 = team ? i1 : i0;
  const int mrb = team ? rb1 : rb0;
  double2 acc[AR][8];
  init_im(acc, M, n, mi0, j0, mrb, jb, true, tr0);
  pipeline<STAGES>(
      j * NS,
      [&](int s, int it) {
        const int64_t k0 = (int64_t)it * W;
        cp_blk<W>(SB(s), A, n, j0, k0, jb, W);
        cp_blk<W>(SA(s, 0), A, n, i0, k0, rb0, W);
        if (AR == 2) cp_blk<W>(SA(s, 1), A, n, i1, k0, rb1, W);
        cp_commit();
      },
      [&](int s, int) { mma_sw<true, true, AR, W>(SA(s, team), SB(s), W, acc, tr0); });
  to_smem(F(1 + team), acc, tr0);
  load_adjU(F(0), A, n, j0, jb);  // C_jj^{-1}
  __syncthreads();
  double2 l[AR][8];
  zero(l);
  mma_sw<true, false, AR>(F(1 + team), F(0), jb, l, tr0);
#pragma unroll
  for (int i = 0; i < AR; ++i)
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
      const int r = fr_row(tr0, i), c = fr_col(jj);
      if (r < mrb && c < jb) A[(mi0 + r) * n + j0 + c] = l[i][jj];
    }
  __syncthreads();
}

// One problem.  The block products stream K slices of width W = 32 / NS through STAGES
// buffer sets (SB, SA0, SA1) of 32 x W values each; the diagonal factorisation, the panel
// finalisation and the inverse columns reuse the same memory as whole 32 x 32 blocks F(0..2).
template <bool INV, int STAGES, int NS, typename MT>
__device__ __forceinline__ void chol_problem(const MT* __restrict__ M, double2* __restrict__ A,
                                             double* __restrict__ logdet,
                                             double2* __restrict__ trace, int* __restrict__ info,
                                             int64_t n, int inv_group) {
  constexpr int W = CB / NS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double2* base = reinterpret_cast<double2*>(smem_raw);
  auto SB = [&](int s) { return base + (3 * s + 0) * CB * W; };
  auto SA = [&](int s, int t) { return base + (3 * s + 1 + t) * CB * W; };
  auto F = [&](int i) { return base + i * CB * CB; };
  __shared__ double s_ld;
  __shared__ int s_bad;
  __shared__ double s_red[2][NT];
  const int nblk = (int)((n + CB - 1) / CB);
  const int w = threadIdx.x >> 5;

  if (threadIdx.x == 0) {
    s_ld = 0.0;
    s_bad = 0;
  }
  // trace of M: the first 64 threads sum with stride 64 and the rest add zeros, so the sums
  // are formed in the order of the two-warp kernel
  double tr = 0, ti = 0;
  if (threadIdx.x < 64)
    for (int64_t i = threadIdx.x; i < n; i += 64) {
      const MT m = M[i * n + i];
      tr += m.x;
      ti += m.y;
    }
  s_red[0][threadIdx.x] = tr;
  s_red[1][threadIdx.x] = ti;
  __syncthreads();

  for (int j = 0; j < nblk; ++j) {
    const int64_t j0 = (int64_t)j * CB;
    const int jb = (int)(CB < (n - j0) ? (int64_t)CB : (n - j0));
    // 1. diagonal block: (I - M)_jj - sum_kb L_j,kb L_j,kb^H, all four warps (one tile row each)
    {
      double2 acc[1][8];
      init_im(acc, M, n, j0, j0, jb, jb, false, w);
      pipeline<STAGES>(
          j * NS,
          [&](int s, int it) {
            cp_blk<W>(SB(s), A, n, j0, (int64_t)it * W, jb, W);
            cp_commit();
          },
          [&](int s, int) { mma_sw<true, true, 1, W>(SB(s), SB(s), W, acc, w); });
      to_smem(F(0), acc, w);
    }
    __syncthreads();
    factor_diag(F(0), jb, &s_ld, &s_bad);
    invert_lower(F(0), F(1), jb);
    store_adjU(F(1), A, n, j0, jb);  // C_jj^{-H} in the upper triangle
    __syncthreads();

    // 2. panel, two row blocks per step, the last one alone when their number is odd:
    // L_i,j = [(I - M)_i,j - sum_kb L_i,kb L_j,kb^H] C_jj^{-H}
    int ib = j + 1;
    for (; ib + 1 < nblk; ib += 2) panel_step<2, STAGES, NS, MT>(M, A, n, j, ib, SB, SA, F);
    if (ib < nblk) panel_step<1, STAGES, NS, MT>(M, A, n, j, ib, SB, SA, F);
  }

  if (INV) {
    for (int j = 0; j < nblk; ++j)
      inverse_column(A, n, j, min(nblk, (j / inv_group + 1) * inv_group), F(0), F(1));
  }

  for (int r = NT / 2; r > 0; r >>= 1) {
    if (threadIdx.x < r) {
      s_red[0][threadIdx.x] += s_red[0][threadIdx.x + r];
      s_red[1][threadIdx.x] += s_red[1][threadIdx.x + r];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *logdet = 2.0 * s_ld;
    *trace = make_double2(s_red[0][0], s_red[1][0]);
    *info = s_bad;
  }
}

// staging bytes: STAGES sets of three 32 x (32 / NS) tiles, at least three whole blocks
template <int STAGES, int NS>
constexpr size_t smem_bytes() {
  return (size_t)3 * CB * CB * sizeof(double2) * (STAGES > NS ? STAGES / NS : 1);
}
template <int STAGES, int NS>
constexpr int min_blocks() {
  return smem_bytes<STAGES, NS>() > 64 * 1024 ? 2 : 4;
}

// M: complex64 (the mixed form) or complex128 (the FP64 form)
template <bool INV, int STAGES, int NS, typename MT = float2>
__global__ void __launch_bounds__(NT, (min_blocks<STAGES, NS>()))
    k_chol_pair(const MT* __restrict__ Mall, double2* __restrict__ Aall,
                double* __restrict__ logdet, double2* __restrict__ trace, int* __restrict__ info,
                int64_t n, int inv_group) {
  const int64_t p = blockIdx.x;
  chol_problem<INV, STAGES, NS, MT>(Mall + p * n * n, Aall + p * n * n, logdet + p, trace + p,
                                    info + p, n, inv_group);
}

}  // namespace p32
