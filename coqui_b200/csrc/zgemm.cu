// Batched complex128 GEMM on the FP64 tensor cores (zgemm.cuh).
//
// CTA tile 64 x 64, 128 x 32 or 32 x 128 complex outputs (the least padding of the shape), four
// warps of 32 x 32 (a 4 x 4 grid of 8 x 8 fragments of mma.sync m8n8k4 FP64; four real
// products per complex one).  K runs in slices of 16: the
// next slice's operand tiles are copied by cp.async while the current one is multiplied
// (two buffers, one barrier per slice).  Shared tiles hold the stored values of op(A) as
// [m][k] and of op(B) as [n][k] (a transposed operand is placed element by element), with the
// XOR swizzle of 16-byte slots used by the factorisation kernels (conflict-free fragment
// reads and copies); conjugation enters as signs of the products.  Each output element sums
// its K terms in increasing k.
#include <algorithm>
#include <type_traits>

#include "zgemm.cuh"

namespace cq {

namespace {

constexpr int TK = 16, NT = 128;

struct ZP {
  int64_t M, N, K;
  double2 alpha, beta;
  int use_beta;
  const double2* A;
  int64_t lda, sA;
  const double2* B;
  int64_t ldb, sB;
  double2* C;
  int64_t ldc, sC;
  const double2* const* Ap;
  const double2* const* Bp;
  double2* const* Cp;
  int64_t b0;
  int a_upper, a_lower, b_lower, b_upper, lower_only, upper_zero;
  int64_t a_mod, a_q0, b_mod, b_q0;
};

__device__ __forceinline__ int swz(int r) { return ((r & 1) << 2) | ((r >> 1) & 3); }
__device__ __forceinline__ int sidx(int r, int c) { return r * TK + (c ^ swz(r)); }

// 16-byte global -> shared asynchronous copy; valid = false zero-fills (no bytes are read)
__device__ __forceinline__ void cp16(double2* dst, const double2* src, bool valid) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}

// One K slice of a TR x 16 tile (rows r = m or n, columns c = k) to shared memory at
// sidx(r, c), TR / 8 elements per thread, asynchronously.  ROW: tile element (r, c) is
// src[(r0 + r) ld + c0 + c]; otherwise src[(c0 + c) ld + r0 + r] (consecutive threads along
// the contiguous index either way); zero unless r0 + r < rmax and c0 + c < cmax.
template <bool ROW, int TR>
__device__ __forceinline__ void cp_tile(double2* S, const double2* __restrict__ src, int64_t ld,
                                        int64_t r0, int64_t c0, int64_t rmax, int64_t cmax) {
#pragma unroll
  for (int u = 0; u < TR * TK / NT; ++u) {
    const int i = threadIdx.x + u * NT;
    const int r = ROW ? (i / TK) : (i % TR), c = ROW ? (i % TK) : (i / TR);
    const bool ok = r0 + r < rmax && c0 + c < cmax;
    cp16(S + sidx(r, c), ok ? src + (ROW ? (r0 + r) * ld + c0 + c : (c0 + c) * ld + r0 + r) : src,
         ok);
  }
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// AN: op(A) = A ('N') or A^H ('C'); BN likewise for B.  The shared tiles hold the stored
// values; conjugation enters as signs: with x, y the stored values and sa, sb = -1 for 'C',
//   Re += xr yr - (sa sb) xi yi,   Im += sb xr yi + sa xi yr.
// The CTA tile is TM = 32 WM rows by TN = 32 (4 / WM) columns, one 32 x 32 block per warp.
template <bool AN, bool BN, int WM>
__global__ void __launch_bounds__(NT, 2) k_zgemm(const __grid_constant__ ZP p) {
  constexpr int WN = 4 / WM, TM = 32 * WM, TN = 32 * WN;
  extern __shared__ __align__(16) double2 zsm[];
  const int64_t b = p.b0 + blockIdx.z;
  const int64_t m0 = (int64_t)blockIdx.y * TM, n0 = (int64_t)blockIdx.x * TN;
  if (p.lower_only && n0 > m0 + TM - 1) return;  // uniform over the CTA
  const double2* A = p.Ap ? p.Ap[b] : p.A + (p.a_mod ? (p.a_q0 + b) % p.a_mod : b) * p.sA;
  const double2* B = p.Bp ? p.Bp[b] : p.B + (p.b_mod ? (p.b_q0 + b) % p.b_mod : b) * p.sB;
  double2* C = p.Cp ? p.Cp[b] : p.C + b * p.sC;

  int64_t klo = 0, khi = p.K;
  if (p.a_upper) klo = max(klo, m0);
  if (p.b_lower) klo = max(klo, n0);
  if (p.a_lower) khi = min(khi, m0 + TM);
  if (p.b_upper) khi = min(khi, n0 + TN);
  klo = klo / TK * TK;
  const bool zero_tile = p.upper_zero && m0 > n0 + TN - 1;  // written as zeros
  const int ns = (khi > klo && !zero_tile) ? (int)((khi - klo + TK - 1) / TK) : 0;

  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, g = l >> 2, q = l & 3;
  const int wm = w / WN, wn = w % WN;
  constexpr double sa = AN ? 1.0 : -1.0, sb = BN ? 1.0 : -1.0, s2 = -sa * sb;
  double cr[4][4][2], ci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;

  // op(A)(m, k): 'N' row m of A; 'C' column m of A.  op(B) kept as [n][k]: 'N' column n of B
  // (transposed placement), 'C' row n of B.
  auto issue = [&](int s) {
    const int64_t k0 = klo + (int64_t)s * TK;
    double2* As = zsm + (s & 1) * (TM + TN) * TK;
    cp_tile<AN, TM>(As, A, p.lda, m0, k0, p.M, p.K);
    cp_tile<!BN, TN>(As + TM * TK, B, p.ldb, n0, k0, p.N, p.K);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if (ns > 0) issue(0);
  for (int s = 0; s < ns; ++s) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();  // slice s is visible, and every warp is done with slice s - 1
    if (s + 1 < ns) issue(s + 1);
    const double2* Xs = zsm + (s & 1) * (TM + TN) * TK;
    const double2* Ys = Xs + TM * TK;
#pragma unroll
    for (int kk = 0; kk < TK / 4; ++kk) {
      const int k = kk * 4 + q;
      double2 x[4], y[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) x[i] = Xs[sidx(32 * wm + 8 * i + g, k)];
#pragma unroll
      for (int j = 0; j < 4; ++j) y[j] = Ys[sidx(32 * wn + 8 * j + g, k)];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(cr[i][j][0], cr[i][j][1], x[i].x, y[j].x);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(cr[i][j][0], cr[i][j][1], s2 * x[i].y, y[j].y);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(ci[i][j][0], ci[i][j][1], sb * x[i].x, y[j].y);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(ci[i][j][0], ci[i][j][1], sa * x[i].y, y[j].x);
    }
  }
  // C = alpha acc + beta C
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t r = m0 + 32 * wm + 8 * i + g, c = n0 + 32 * wn + 8 * j + 2 * q + e;
        if (r >= p.M || c >= p.N) continue;
        const double ar = cr[i][j][e], ai = ci[i][j][e];
        double2 v = make_double2(p.alpha.x * ar - p.alpha.y * ai, p.alpha.x * ai + p.alpha.y * ar);
        double2* dst = C + r * p.ldc + c;
        if (p.use_beta) {
          const double2 o = *dst;
          v.x += p.beta.x * o.x - p.beta.y * o.y;
          v.y += p.beta.x * o.y + p.beta.y * o.x;
        }
        *dst = v;
      }
}

template <bool AN, bool BN, int WM>
void launch(const ZP& base, int64_t batch, cudaStream_t s) {
  constexpr int TM = 32 * WM, TN = 32 * (4 / WM);
  auto fn = k_zgemm<AN, BN, WM>;
  const int smem = 2 * (TM + TN) * TK * (int)sizeof(double2);
  static bool attr[64] = {};
  int dev = 0;
  CQ_CHECK_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && !attr[dev]) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr[dev] = true;
  }
  const int64_t gx = (base.N + TN - 1) / TN, gy = (base.M + TM - 1) / TM;
  CQ_REQUIRE(gx <= 2147483647 && gy <= 65535, COQUI_B200_EINVAL, "zgemm: matrix too large");
  for (int64_t b0 = 0; b0 < batch; b0 += 65535) {
    ZP p = base;
    p.b0 = b0;
    const int64_t nb = std::min<int64_t>(65535, batch - b0);
    fn<<<dim3((unsigned)gx, (unsigned)gy, (unsigned)nb), NT, smem, s>>>(p);
    count_launch();
    CQ_CHECK_CUDA(cudaGetLastError());
  }
}

}  // namespace

void zgemm(const ZgemmArgs& a, cudaStream_t s) {
  CQ_REQUIRE((a.opA == 'N' || a.opA == 'C') && (a.opB == 'N' || a.opB == 'C'), COQUI_B200_EINVAL,
             "zgemm: op must be N or C");
  CQ_REQUIRE(a.M >= 0 && a.N >= 0 && a.K >= 0 && a.batch >= 0, COQUI_B200_EINVAL,
             "zgemm: negative size");
  if (a.M == 0 || a.N == 0 || a.batch == 0) return;
  ZP p{};
  p.M = a.M;
  p.N = a.N;
  p.K = a.K;
  p.alpha = a.alpha;
  p.beta = a.beta;
  p.use_beta = (a.beta.x != 0.0 || a.beta.y != 0.0) ? 1 : 0;
  p.A = a.A;
  p.lda = a.lda;
  p.sA = a.sA;
  p.B = a.B;
  p.ldb = a.ldb;
  p.sB = a.sB;
  p.C = a.C;
  p.ldc = a.ldc;
  p.sC = a.sC;
  p.Ap = a.Ap;
  p.Bp = a.Bp;
  p.Cp = a.Cp;
  p.a_upper = a.a_upper;
  p.a_lower = a.a_lower;
  p.b_lower = a.b_lower;
  p.b_upper = a.b_upper;
  p.lower_only = a.lower_only;
  p.upper_zero = a.upper_zero;
  p.a_mod = a.a_mod;
  p.a_q0 = a.a_q0;
  p.b_mod = a.b_mod;
  p.b_q0 = a.b_q0;
  // CTA tile 64 x 64, 128 x 32 or 32 x 128: the least padding of M x N (64 x 64 on ties)
  auto padded = [&](int64_t tm, int64_t tn) {
    return ((a.M + tm - 1) / tm * tm) * ((a.N + tn - 1) / tn * tn);
  };
  int wm = 2;
  int64_t best = padded(64, 64);
  if (padded(128, 32) < best) wm = 4, best = padded(128, 32);
  if (padded(32, 128) < best) wm = 1;
  const bool an = a.opA == 'N', bn = a.opB == 'N';
  auto go = [&](auto an_t, auto bn_t) {
    constexpr bool AN = decltype(an_t)::value, BN = decltype(bn_t)::value;
    if (wm == 4) launch<AN, BN, 4>(p, a.batch, s);
    else if (wm == 1) launch<AN, BN, 1>(p, a.batch, s);
    else launch<AN, BN, 2>(p, a.batch, s);
  };
  using T = std::true_type;
  using F = std::false_type;
  if (an && bn) go(T{}, T{});
  else if (an) go(T{}, F{});
  else if (bn) go(F{}, T{});
  else go(F{}, F{});
}

}  // namespace cq
