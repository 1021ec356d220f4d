// Batched FP64 Cholesky factorisation, log-determinant and triangular inverse of
// A = I - M (one CTA per Np x Np problem), the factorisation step of the Dyson solve.
//
//   A = C C^H (C lower, FP64), logdet = 2 sum_i ln C_ii, trace = sum_i M_ii,
//   optional DH = C^{-H} - I (upper triangular, FP64) for W = L (D + D^H + D^H D) L^H.
//
// Blocked algorithm (chol_blk.cuh), by default in left-looking order: block column j is
// A_ij - sum_{k<j} L_ik L_jk^H formed from I - M and the finished columns, the diagonal block
// is factored and inverted in shared memory and the panel below is L_ib = (...) C_jj^{-H}.
// COQUI_B200_CHOL_ORDER=right selects the right-looking order (the trailing lower triangle
// gets A_ik -= L_ij L_kj^H after every column), which subtracts the same products in the same
// order and gives identical results with more memory traffic.  The inverse is formed block column by block column:
// X_ij = -C_ii^{-1} sum_{k=j}^{i-1} C_ik X_kj.  The 32 x 32 block products run on the FP64
// tensor cores (mma.sync m8n8k4, four real products per complex one; each of the two warps
// holds a 16 x 32 accumulator as 8 x 8 fragments), operands staged in shared memory; the
// CUDA-core FMA form (4 x 4 register tiles) is kept behind CHOL_FMA for comparison.  A = I - M
// is read from M in the first block column (A holds only FP64 blocks written by the
// factorisation); D^H is written out by a separate element-wise kernel.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <string>
#include <vector>

#include "chol.cuh"

namespace cq {

namespace {

__device__ __forceinline__ double2 cmul_(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc_(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 conj_(double2 a) { return make_double2(a.x, -a.y); }

// The blocked algorithm (chol_blk.cuh) with 32 x 32 blocks and 64 threads: two staging blocks
// (34 KB) per problem let six problems share an SM, so that one problem's barriers and loads
// overlap the others' FP64 arithmetic.  (64 x 64 blocks halve the block traffic per flop but
// leave one problem per SM; measured slower.)
namespace b32 {
#ifdef CHOL_FMA
constexpr bool DMMA = false;
#else
constexpr bool DMMA = true;
#endif
constexpr int CB = 32, RT = 4, CTT = 4, TWR = CB / RT, TWC = CB / CTT, CT = TWR * TWC,
              PITCH = CB + 1, MINB = 6;
constexpr int AR = DMMA ? 2 : RT, AC = DMMA ? 8 : CTT;
static_assert(!DMMA || (CB == 32 && CT == 64), "DMMA tiles: 32-blocks, two warps");
#include "chol_blk.cuh"
}  // namespace b32

// Four-warp left-looking kernel (two panel row blocks per step, cp.async staging): the same
// arithmetic as b32::k_chol_inv_left with less block traffic per product.
#include "chol_pair.cuh"

// Problems of different sizes in one launch (one CTA each, 32-blocks).
template <bool LEFT>
__global__ void __launch_bounds__(b32::CT, b32::MINB) k_chol_inv_grouped(const CholProblem* __restrict__ probs,
                                                                 double* __restrict__ logdet,
                                                                 double2* __restrict__ trace,
                                                                 int* __restrict__ info,
                                                                 int inv_group) {
  const CholProblem pr = probs[blockIdx.x];
  if constexpr (LEFT)
    b32::chol_inv_problem_left<true>(pr.M, pr.A, logdet + blockIdx.x, trace + blockIdx.x,
                                     info + blockIdx.x, pr.n, inv_group);
  else
    b32::chol_inv_problem<true>(pr.M, pr.A, logdet + blockIdx.x, trace + blockIdx.x,
                                info + blockIdx.x, pr.n, inv_group);
}

// ---- tiled factorisation (several CTAs per problem) ----
// Problems come in runs of equal size; a problem's matrices are taken from the table, or
// (table == nullptr, one run) at base + p * stride.
constexpr int kMaxRuns = 64;
struct TiledRuns {
  int nrun;
  int64_t n[kMaxRuns];
  int first[kMaxRuns];
  int count[kMaxRuns];
  const float2* M0;
  double2* A0;
  int64_t stride;
};
constexpr int kTiledG = (int)(kInvGroup / b32::CB);  // blocks per diagonal inverse group

// Block columns are taken in groups of kTiledCols: for each column of a group, its blocks are
// updated by the group's earlier columns, then its diagonal block and panel are factored; then
// the trailing blocks get the whole group's updates in one pass.  The products and their
// order are those of one column at a time; the trailing matrix is read and written once per
// group.
constexpr int kTiledCols = 8;

// work items of one launch: kind 0 diagonal block j (one per problem), 1 panel blocks below
// it, 2 trailing blocks (i, k) with j + cols <= k <= i, updated by the block columns j ..
// j + cols - 1, 3 inverse columns (all columns that have a block below them in their group;
// j is not used), 4 the blocks (i, j + cols), i >= j + cols, of block column j + cols updated
// by the columns j .. j + cols - 1.
__host__ __device__ inline int64_t tiled_items(int kind, int64_t nblk, int j, int cols) {
  const int64_t m = nblk - j - 1;
  switch (kind) {
    case 0: return nblk > j ? 1 : 0;
    case 1: return m > 0 ? m : 0;
    case 2: {
      const int64_t t = nblk - j - cols;
      return t > 0 ? t * (t + 1) / 2 : 0;
    }
    case 4: {
      const int64_t t = nblk - j - cols;
      return t > 0 ? t : 0;
    }
    default: return nblk - (nblk + kTiledG - 1) / kTiledG;
  }
}

__global__ void __launch_bounds__(b32::CT, b32::MINB)
    k_chol_tiled(const CholProblem* __restrict__ probs, const __grid_constant__ TiledRuns R, int kind,
                 int j, int cols, double* __restrict__ logdet, int* __restrict__ info) {
  int64_t idx = blockIdx.x, local = 0, nblk = 0;
  int p = -1;
  for (int r = 0; r < R.nrun; ++r) {
    const int64_t nb = (R.n[r] + b32::CB - 1) / b32::CB;
    const int64_t per = tiled_items(kind, nb, j, cols), tot = per * R.count[r];
    if (idx < tot) {
      p = R.first[r] + (int)(idx / per);
      local = idx % per;
      nblk = nb;
      break;
    }
    idx -= tot;
  }
  if (p < 0) return;  // uniform over the CTA
  double2* A = probs ? probs[p].A : R.A0 + p * R.stride;
  const float2* M = probs ? probs[p].M : R.M0 + p * R.stride;
  const int64_t n = probs ? probs[p].n : R.n[0];
  if (kind == 0) {
    b32::tiled_diag(M, A, n, j, logdet + p, info + p);
  } else if (kind == 1) {
    b32::tiled_panel(M, A, n, j, j + 1 + (int)local);
  } else if (kind == 2) {  // local -> (i', k'), 0 <= k' <= i'
    int64_t a = (int64_t)((sqrt(8.0 * (double)local + 1.0) - 1.0) * 0.5);
    while ((a + 1) * (a + 2) / 2 <= local) ++a;
    while (a * (a + 1) / 2 > local) --a;
    const int64_t b = local - a * (a + 1) / 2;
    b32::tiled_update_cols(M, A, n, j, cols, j + cols + (int)a, j + cols + (int)b);
  } else if (kind == 4) {
    b32::tiled_update_cols(M, A, n, j, cols, j + cols + (int)local, j + cols);
  } else {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* S0 = reinterpret_cast<double2*>(smem_raw);
    double2* S1 = S0 + b32::CB * b32::PITCH;
    const int jj = (int)(local + local / (kTiledG - 1));
    b32::inverse_column(A, n, jj, (int)min(nblk, (int64_t)(jj / kTiledG + 1) * kTiledG), S0, S1);
  }
}

// trace = sum_i M_ii, logdet = 0, info = 0 per problem
__global__ void k_tiled_init(const CholProblem* __restrict__ probs, const __grid_constant__ TiledRuns R,
                             double* __restrict__ logdet, double2* __restrict__ trace,
                             int* __restrict__ info) {
  __shared__ double red[2][256];
  const int p = blockIdx.x;
  const float2* M = probs ? probs[p].M : R.M0 + p * R.stride;
  const int64_t n = probs ? probs[p].n : R.n[0];
  double tr = 0, ti = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const float2 m = M[i * n + i];
    tr += m.x;
    ti += m.y;
  }
  red[0][threadIdx.x] = tr;
  red[1][threadIdx.x] = ti;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      red[0][threadIdx.x] += red[0][threadIdx.x + w];
      red[1][threadIdx.x] += red[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    trace[p] = make_double2(red[0][0], red[1][0]);
    logdet[p] = 0.0;
    info[p] = 0;
  }
}

void run_tiled(const CholProblem* t, const TiledRuns& R, int64_t np, double* logdet, double2* trace,
               int* info, cudaStream_t s) {
  k_tiled_init<<<(unsigned)np, 256, 0, s>>>(t, R, logdet, trace, info);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  const size_t smem = (size_t)2 * b32::CB * b32::PITCH * sizeof(double2);
  static bool set = false;
  if (!set) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(k_chol_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    set = true;
  }
  int64_t maxblk = 0;
  for (int r = 0; r < R.nrun; ++r) maxblk = std::max<int64_t>(maxblk, (R.n[r] + b32::CB - 1) / b32::CB);
  auto go = [&](int kind, int j, int cols) {
    int64_t grid = 0;
    for (int r = 0; r < R.nrun; ++r)
      grid += tiled_items(kind, (R.n[r] + b32::CB - 1) / b32::CB, j, cols) * R.count[r];
    if (grid == 0) return;
    CQ_REQUIRE(grid <= 2147483647, COQUI_B200_EINVAL, "tiled Cholesky: too many blocks");
    k_chol_tiled<<<(unsigned)grid, b32::CT, smem, s>>>(t, R, kind, j, cols, logdet, info);
    count_launch();
    CQ_CHECK_CUDA(cudaGetLastError());
  };
  for (int j = 0; j < maxblk; j += kTiledCols) {
    const int g = (int)std::min<int64_t>(kTiledCols, maxblk - j);
    for (int c = 0; c < g; ++c) {
      if (c > 0) go(4, j, c);  // column j + c by the group's columns j .. j + c - 1
      go(0, j + c, 0);
      go(1, j + c, 0);
    }
    go(2, j, g);  // the trailing blocks by the whole group
  }
  go(3, 0, 0);
}

// Form of the one-CTA factorisation, COQUI_B200_CHOL_ORDER: "pair" (default: four warps,
// two panel row blocks per step, double-buffered half-width K slices), "pair1" (the same with
// whole blocks copied and then used), "pair2" (double-buffered whole blocks), "left" (two
// warps, left-looking), "right" (two warps, right-looking).  All give identical results.
enum class CholForm { kPair, kPair1, kPair2, kLeft, kRight };
CholForm chol_form() {
  const char* v = std::getenv("COQUI_B200_CHOL_ORDER");
  if (!v || !v[0]) return CholForm::kPair;
  const std::string f(v);
  if (f == "right") return CholForm::kRight;
  if (f == "left") return CholForm::kLeft;
  if (f == "pair2") return CholForm::kPair2;
  if (f == "pair1") return CholForm::kPair1;
  return CholForm::kPair;
}
bool chol_left_looking() { return chol_form() != CholForm::kRight; }

// k_chol_inv<INV> of the block size chosen for n; the inverse is formed within diagonal groups
// of inv_cols columns (a multiple of 64).
template <bool INV>
void launch_factor(const float2* M, double2* A, double* logdet, double2* trace, int* info,
                   int64_t n, int64_t nprob, int64_t inv_cols, cudaStream_t s) {
  auto go = [&](auto kern, int cb, int ct, int pitch) {
    const size_t smem = (size_t)2 * cb * pitch * sizeof(double2);
    CQ_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int groups = (int)std::min<int64_t>(inv_cols / cb, 1 << 30);
    kern<<<(unsigned)nprob, ct, smem, s>>>(M, A, logdet, trace, info, n, groups);
    count_launch();
    CQ_CHECK_CUDA(cudaGetLastError());
  };
  auto go_pair = [&](auto kern, size_t smem) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int groups = (int)std::min<int64_t>(inv_cols / p32::CB, 1 << 30);
    kern<<<(unsigned)nprob, p32::NT, smem, s>>>(M, A, logdet, trace, info, n, groups);
    count_launch();
    CQ_CHECK_CUDA(cudaGetLastError());
  };
  switch (chol_form()) {
    case CholForm::kPair: go_pair(p32::k_chol_pair<INV, 2, 2>, p32::smem_bytes<2, 2>()); break;
    case CholForm::kPair1: go_pair(p32::k_chol_pair<INV, 1, 1>, p32::smem_bytes<1, 1>()); break;
    case CholForm::kPair2: go_pair(p32::k_chol_pair<INV, 2, 1>, p32::smem_bytes<2, 1>()); break;
    case CholForm::kLeft: go(b32::k_chol_inv_left<INV>, b32::CB, b32::CT, b32::PITCH); break;
    default: go(b32::k_chol_inv<INV>, b32::CB, b32::CT, b32::PITCH); break;
  }
}

// grouped Z = X^H - I, blockIdx.y = problem
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
  const int64_t total = Np * Np * nprob;
  const int64_t all = (int64_t)1 << 40;  // inverse over the whole matrix
  if (Z) {
    launch_factor<true>(M, A, logdet, trace, info, Np, nprob, all, s);
    k_chol_final<<<grid_for(total, 256), 256, 0, s>>>(A, Z, Np, total);
    count_launch();
    CQ_CHECK_CUDA(cudaGetLastError());
  } else {
    launch_factor<false>(M, A, logdet, trace, info, Np, nprob, all, s);
  }
}

void launch_chol_group_inv(const float2* M, double2* A, double* logdet, double2* trace, int* info,
                           int64_t Np, int64_t nprob, cudaStream_t s) {
  launch_factor<true>(M, A, logdet, trace, info, Np, nprob, kInvGroup, s);
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

bool chol_prefer_tiled(const std::vector<int64_t>& sizes) {
  // COQUI_B200_CHOL_TILED=1 / 0 forces the choice (for problems above one inverse group)
  const char* force = std::getenv("COQUI_B200_CHOL_TILED");
  const int64_t nmax0 = sizes.empty() ? 0 : *std::max_element(sizes.begin(), sizes.end());
  if (force && (force[0] == '0' || force[0] == '1'))
    return force[0] == '1' && nmax0 >= 4 * b32::CB;
  // one CTA per problem: the makespan is at least the largest problem's time; spreading each
  // problem over many CTAs pays when the whole set would otherwise finish sooner than that
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double total = 0, mx = 0;
  for (int64_t n : sizes) {
    const double c = (double)n * n * n;
    total += c;
    mx = std::max(mx, c);
  }
  const int64_t nmax = sizes.empty() ? 0 : *std::max_element(sizes.begin(), sizes.end());
  return nmax >= 4 * b32::CB && total / (double)chol_wave_size() < mx;
}

void launch_chol_inv_c128(const double2* M, double2* A, double* logdet, double2* trace, int* info,
                          int64_t Np, int64_t nprob, cudaStream_t s) {
  auto kern = p32::k_chol_pair<true, 2, 2, double2>;
  const size_t smem = p32::smem_bytes<2, 2>();
  CQ_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CQ_REQUIRE(nprob <= 2147483647, COQUI_B200_EINVAL, "chol: too many problems");
  kern<<<(unsigned)nprob, p32::NT, smem, s>>>(M, A, logdet, trace, info, Np, 1 << 30);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

// Z = U - I from the upper triangle U of A (complex128), zero below the diagonal
__global__ void k_upper_minus_eye(const double2* __restrict__ A, double2* __restrict__ Z, int64_t n,
                                  int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i % (n * n), r = e / n, c = e % n;
    double2 z = make_double2(0.0, 0.0);
    if (c >= r) {
      z = A[i];
      if (c == r) z.x -= 1.0;
    }
    Z[i] = z;
  }
}

void launch_upper_minus_eye(const double2* A, double2* Z, int64_t Np, int64_t nprob,
                            cudaStream_t s) {
  const int64_t total = Np * Np * nprob;
  k_upper_minus_eye<<<grid_for(total, 256), 256, 0, s>>>(A, Z, Np, total);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

int64_t chol_wave_size() {
  int dev = 0, sms = 148, per_sm = 0;
  CQ_CHECK_CUDA(cudaGetDevice(&dev));
  CQ_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  size_t smem = (size_t)2 * b32::CB * b32::PITCH * sizeof(double2);
  int threads = b32::CT;
  const void* kern = nullptr;
  switch (chol_form()) {
    case CholForm::kPair:
      kern = (const void*)p32::k_chol_pair<true, 2, 2>, smem = p32::smem_bytes<2, 2>();
      threads = p32::NT;
      break;
    case CholForm::kPair1:
      kern = (const void*)p32::k_chol_pair<true, 1, 1>, smem = p32::smem_bytes<1, 1>();
      threads = p32::NT;
      break;
    case CholForm::kPair2:
      kern = (const void*)p32::k_chol_pair<true, 2, 1>, smem = p32::smem_bytes<2, 1>();
      threads = p32::NT;
      break;
    case CholForm::kLeft: kern = (const void*)b32::k_chol_inv_left<true>; break;
    default: kern = (const void*)b32::k_chol_inv<true>; break;
  }
  CQ_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CQ_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
  return (int64_t)sms * std::max(per_sm, 1);
}

void launch_chol_tiled_strided(const float2* M, double2* A, double* logdet, double2* trace,
                               int* info, int64_t Np, int64_t nprob, cudaStream_t s) {
  CQ_REQUIRE(nprob <= 2147483647, COQUI_B200_EINVAL, "tiled Cholesky: too many problems");
  TiledRuns R{};
  R.nrun = 1;
  R.n[0] = Np;
  R.first[0] = 0;
  R.count[0] = (int)nprob;
  R.M0 = M;
  R.A0 = A;
  R.stride = Np * Np;
  run_tiled(nullptr, R, nprob, logdet, trace, info, s);
}

void launch_chol_tiled(const std::vector<CholProblem>& probs, DevBuf<unsigned char>& table,
                       double* logdet, double2* trace, int* info, cudaStream_t s) {
  if (probs.empty()) return;
  const int64_t np = (int64_t)probs.size();
  TiledRuns R{};
  for (int64_t p = 0; p < np; ++p) {
    if (R.nrun > 0 && R.n[R.nrun - 1] == probs[p].n) {
      ++R.count[R.nrun - 1];
      continue;
    }
    CQ_REQUIRE(R.nrun < kMaxRuns, COQUI_B200_EINVAL, "tiled Cholesky: too many problem sizes");
    R.n[R.nrun] = probs[p].n;
    R.first[R.nrun] = (int)p;
    R.count[R.nrun] = 1;
    ++R.nrun;
  }
  // largest problems first within every launch (the work items are decoded run by run)
  std::vector<int> ord(R.nrun);
  for (int r = 0; r < R.nrun; ++r) ord[r] = r;
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return R.n[x] > R.n[y]; });
  TiledRuns S = R;
  for (int r = 0; r < R.nrun; ++r) {
    S.n[r] = R.n[ord[r]];
    S.first[r] = R.first[ord[r]];
    S.count[r] = R.count[ord[r]];
  }
  table.ensure(np * sizeof(CholProblem));
  CQ_CHECK_CUDA(cudaMemcpyAsync(table.p, probs.data(), np * sizeof(CholProblem),
                                cudaMemcpyHostToDevice, s));
  run_tiled((const CholProblem*)table.p, S, np, logdet, trace, info, s);
}

void launch_chol_inv_grouped(const std::vector<CholProblem>& probs, DevBuf<unsigned char>& table,
                             double* logdet, double2* trace, int* info, cudaStream_t s,
                             bool group_inverse) {
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
  const size_t smem = (size_t)2 * b32::CB * b32::PITCH * sizeof(double2);
  const int inv_group = group_inverse ? (int)(kInvGroup / b32::CB) : (1 << 30);
  auto go = [&](auto kern) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)np, b32::CT, smem, s>>>(t, logdet, trace, info, inv_group);
  };
  if (chol_left_looking())
    go(k_chol_inv_grouped<true>);
  else
    go(k_chol_inv_grouped<false>);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  if (group_inverse) return;
  k_chol_final_grouped<<<dim3(gx, (unsigned)np), 256, 0, s>>>(t);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

}  // namespace cq
