// Split-TF32 complex GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// C[b] (M x N, complex64) = opA(A[b]) * B[b], B given transposed: B[b](k, n) = Bt[b][n][k]
// ("NT" form), A and Bt row-major complex64 or complex128, optional conjugation of either.
//
// Complex -> real: with A_r = [Re a_0, Im a_0, Re a_1, Im a_1, ...] (the interleaved
// storage of an A row) and the realified B rows
//     row 2n   = [Re b_0n, -Im b_0n, Re b_1n, -Im b_1n, ...]
//     row 2n+1 = [Im b_0n,  Re b_0n, Im b_1n,  Re b_1n, ...]
// the real product A_r B_r^T has columns (2n, 2n+1) = (Re c_mn, Im c_mn), i.e. it is C in
// interleaved complex storage.  Each real operand x is split x = hi + lo with hi, lo TF32
// (hi = rna(x), lo = rna(x - hi)); hi*hi + hi*lo + lo*hi accumulate in FP32 in TMEM.
//
// CTA tile: 128 rows x BNC complex columns (UMMA M = 128, N = 2 BNC), 16 complex (32 real)
// of K per pipeline stage = one 128-byte swizzle row.  Warps 0-3 stage operands (global ->
// registers -> split -> swizzled st.shared) and later drain TMEM; warp 4 allocates TMEM and
// one of its lanes issues the MMAs.  Waits are bounded by a 2 s global-timer budget that sets
// an error flag instead of hanging.
#include <cstdint>

#include "kernels.cuh"
#include "tc_gemm.cuh"

namespace cq {

namespace {

__device__ int g_tc_error = 0;

constexpr int kBM = 128;
constexpr int kBKR = 32;  // real K per stage (128 bytes of fp32)
constexpr int kStages = 2;
constexpr int kProducers = 128;
constexpr int kThreads = 160;

template <int BNC> struct TileCfg {
  static constexpr int NR = 2 * BNC;                   // UMMA N (real columns)
  static constexpr int A_PLANE = kBM * 128;            // bytes of one A plane
  static constexpr int B_PLANE = NR * 128;             // bytes of one B plane
  static constexpr int STAGE = 2 * A_PLANE + 2 * B_PLANE;
  static constexpr int SMEM = kStages * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  static constexpr int TMEM_COLS = NR;                 // 64, 128 or 256
  // kind::tf32 dense, F32 accumulate, K-major A and B, M = 128, N = NR
  static constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) |
                                    ((uint32_t)(NR >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
};

struct TcParams {
  const void* A;
  const void* Bt;
  float2* C;
  int64_t M, N, K;
  int64_t lda, ldb, ldc;
  int64_t sA, sB, sC;
  int a64, b64;  // element type is complex128
  int conj_a, conj_b;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" ::"r"(bar) : "memory");
}

// Bounded wait for the phase with the given parity; returns false (and flags) on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  while (true) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (global_ns() - t0 > 2000000000ull) {
      atomicExch(&g_tc_error, 1);
      return false;
    }
  }
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// split x (float or double) into TF32 hi + lo
__device__ __forceinline__ void split2(double x, uint32_t& hi, uint32_t& lo) {
  const float xf = (float)x;
  hi = to_tf32(xf);
  lo = to_tf32((float)(x - (double)__uint_as_float(hi)));
}
__device__ __forceinline__ void split2(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c,
                                             uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c),
               "r"(d)
               : "memory");
}

// byte offset of 16-byte chunk `chunk` (0..7) of row `row` in a 128B-swizzled K-major tile
__device__ __forceinline__ uint32_t sw128(int row, int chunk) {
  return (uint32_t)(row * 128 + ((chunk ^ (row & 7)) << 4));
}

__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                         uint32_t acc) {
  asm volatile(
      "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p; }"
      ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// load two consecutive complex values (k, k+1) of a row as doubles; zero outside [0, kmax)
template <bool C64>
__device__ __forceinline__ void load_pair(const void* base, int64_t off, int64_t k, int64_t kmax,
                                          double v[4]) {
  if (C64) {
    const float2* p = reinterpret_cast<const float2*>(base) + off;
    if (k + 1 < kmax && ((off & 1) == 0)) {
      const float4 q = *reinterpret_cast<const float4*>(p);
      v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    } else {
      float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
      if (k < kmax) a = p[0];
      if (k + 1 < kmax) b = p[1];
      v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
  } else {
    const double2* p = reinterpret_cast<const double2*>(base) + off;
    double2 a = make_double2(0, 0), b = make_double2(0, 0);
    if (k < kmax) a = p[0];
    if (k + 1 < kmax) b = p[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
}

template <int BNC, bool A64, bool B64>
__device__ __forceinline__ void stage_tile(const TcParams& p, int64_t bz, int64_t m0, int64_t n0,
                                           int64_t k0c, uint32_t sA_hi, uint32_t sA_lo,
                                           uint32_t sB_hi, uint32_t sB_lo) {
  const int t = threadIdx.x;  // 0..127
  const double ca = p.conj_a ? -1.0 : 1.0, cb = p.conj_b ? -1.0 : 1.0;
  // A: 128 rows x 8 chunks (2 complex each)
#pragma unroll 2
  for (int i = t; i < kBM * 8; i += kProducers) {
    const int r = i >> 3, c = i & 7;
    const int64_t m = m0 + r, k = k0c + 2 * c;
    double v[4] = {0, 0, 0, 0};
    if (m < p.M) load_pair<!A64>(p.A, bz * p.sA + m * p.lda + k, k, p.K, v);
    v[1] *= ca;
    v[3] *= ca;
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) split2(v[j], h[j], l[j]);
    const uint32_t off = sw128(r, c);
    st_shared_v4(sA_hi + off, h[0], h[1], h[2], h[3]);
    st_shared_v4(sA_lo + off, l[0], l[1], l[2], l[3]);
  }
  // B: BNC complex rows x 8 chunks -> realified rows 2n, 2n+1
#pragma unroll 2
  for (int i = t; i < BNC * 8; i += kProducers) {
    const int r = i >> 3, c = i & 7;
    const int64_t n = n0 + r, k = k0c + 2 * c;
    double v[4] = {0, 0, 0, 0};
    if (n < p.N) load_pair<!B64>(p.Bt, bz * p.sB + n * p.ldb + k, k, p.K, v);
    const double br0 = v[0], bi0 = cb * v[1], br1 = v[2], bi1 = cb * v[3];
    // row 2r: (br, -bi) pairs; row 2r+1: (bi, br) pairs
    const double e0[4] = {br0, -bi0, br1, -bi1};
    const double e1[4] = {bi0, br0, bi1, br1};
    uint32_t h0[4], l0[4], h1[4], l1[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      split2(e0[j], h0[j], l0[j]);
      split2(e1[j], h1[j], l1[j]);
    }
    const uint32_t o0 = sw128(2 * r, c), o1 = sw128(2 * r + 1, c);
    st_shared_v4(sB_hi + o0, h0[0], h0[1], h0[2], h0[3]);
    st_shared_v4(sB_lo + o0, l0[0], l0[1], l0[2], l0[3]);
    st_shared_v4(sB_hi + o1, h1[0], h1[1], h1[2], h1[3]);
    st_shared_v4(sB_lo + o1, l1[0], l1[1], l1[2], l1[3]);
  }
}

template <int BNC, bool A64, bool B64>
__global__ void __launch_bounds__(kThreads, 1) k_tc_cgemm(TcParams p) {
  using Cfg = TileCfg<BNC>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * Cfg::STAGE);
  // bars[0..1] full, bars[2..3] empty, bars[4] accumulator ready; bars[5] holds the TMEM base
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 5);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t bz = blockIdx.z;
  const int64_t m0 = (int64_t)blockIdx.y * kBM, n0 = (int64_t)blockIdx.x * BNC;
  const int nkb = (int)((p.K + 15) / 16);

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&bars[s]), kProducers);
      mbar_init(smem_u32(&bars[kStages + s]), 1);
    }
    mbar_init(smem_u32(&bars[4]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 4) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"((uint32_t)Cfg::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  bool ok = true;
  if (warp < 4) {
    // ---------------- producers ----------------
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % kStages;
      const uint32_t ph = (uint32_t)(kb / kStages) & 1u;
      if (!mbar_wait(smem_u32(&bars[kStages + s]), ph ^ 1u)) { ok = false; break; }
      unsigned char* st = smem + s * Cfg::STAGE;
      const uint32_t a_hi = smem_u32(st), a_lo = a_hi + Cfg::A_PLANE;
      const uint32_t b_hi = a_lo + Cfg::A_PLANE, b_lo = b_hi + Cfg::B_PLANE;
      stage_tile<BNC, A64, B64>(p, bz, m0, n0, (int64_t)kb * 16, a_hi, a_lo, b_hi, b_lo);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(smem_u32(&bars[s]));
    }
    // ---------------- epilogue ----------------
    if (ok && mbar_wait(smem_u32(&bars[4]), 0u)) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int r = warp * 32 + lane;
      const int64_t m = m0 + r;
      float2* crow = p.C + bz * p.sC + m * p.ldc;
      const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
      for (int j = 0; j < Cfg::NR / 32; ++j) {
        uint32_t v[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
            "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
            "%28, %29, %30, %31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
              "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
              "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
              "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
              "=r"(v[31])
            : "r"(trow + (uint32_t)(j * 32)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (m < p.M) {
          const int64_t nb0 = n0 + j * 16;
          const bool vec = ((((uintptr_t)(crow + nb0)) & 15) == 0) && (nb0 + 16 <= p.N);
          if (vec) {
            float4* dst = reinterpret_cast<float4*>(crow + nb0);
#pragma unroll
            for (int q = 0; q < 8; ++q)
              dst[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                                   __uint_as_float(v[4 * q + 2]), __uint_as_float(v[4 * q + 3]));
          } else {
#pragma unroll
            for (int q = 0; q < 16; ++q)
              if (nb0 + q < p.N)
                crow[nb0 + q] = make_float2(__uint_as_float(v[2 * q]), __uint_as_float(v[2 * q + 1]));
          }
        }
      }
    }
  } else if (lane == 0) {
    // ---------------- MMA issuer (warp 4, one lane) ----------------
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % kStages;
      const uint32_t ph = (uint32_t)(kb / kStages) & 1u;
      if (!mbar_wait(smem_u32(&bars[s]), ph)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_hi = smem_u32(smem + s * Cfg::STAGE), a_lo = a_hi + Cfg::A_PLANE;
      const uint32_t b_hi = a_lo + Cfg::A_PLANE, b_lo = b_hi + Cfg::B_PLANE;
#pragma unroll
      for (int kk = 0; kk < kBKR / 8; ++kk) {
        const uint32_t o = (uint32_t)kk * 32;  // 8 tf32 = 32 bytes along K
        const uint64_t ah = make_desc(a_hi + o), al = make_desc(a_lo + o);
        const uint64_t bh = make_desc(b_hi + o), bl = make_desc(b_lo + o);
        const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
        mma_tf32(tmem, al, bh, Cfg::IDESC, acc);
        mma_tf32(tmem, ah, bl, Cfg::IDESC, 1u);
        mma_tf32(tmem, ah, bh, Cfg::IDESC, 1u);
      }
      mma_commit(smem_u32(&bars[kStages + s]));  // frees the stage once these MMAs retire
    }
    if (ok) mma_commit(smem_u32(&bars[4]));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 4) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)Cfg::TMEM_COLS)
                 : "memory");
  }
}

template <int BNC, bool A64, bool B64>
void launch_tc(const TcParams& p, int64_t batch, cudaStream_t s) {
  using Cfg = TileCfg<BNC>;
  auto fn = k_tc_cgemm<BNC, A64, B64>;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
    attr_set[dev] = true;
  }
  for (int64_t b0 = 0; b0 < batch; b0 += 65535) {
    TcParams q = p;
    const int64_t nb = std::min<int64_t>(65535, batch - b0);
    q.A = (const unsigned char*)p.A + b0 * p.sA * (p.a64 ? 16 : 8);
    q.Bt = (const unsigned char*)p.Bt + b0 * p.sB * (p.b64 ? 16 : 8);
    q.C = p.C + b0 * p.sC;
    dim3 grid((unsigned)((p.N + BNC - 1) / BNC), (unsigned)((p.M + kBM - 1) / kBM), (unsigned)nb);
    fn<<<grid, kThreads, Cfg::SMEM, s>>>(q);
    count_launch();
    CQ_CHECK_CUDA(cudaGetLastError());
  }
}

template <bool A64, bool B64>
void dispatch_n(const TcParams& p, int64_t batch, cudaStream_t s) {
  if (p.N >= 128)
    launch_tc<128, A64, B64>(p, batch, s);
  else if (p.N > 32)
    launch_tc<64, A64, B64>(p, batch, s);
  else
    launch_tc<32, A64, B64>(p, batch, s);
}

}  // namespace

void tc_cgemm_nt(const void* A, bool a_c128, bool conj_a, int64_t lda, int64_t sA, const void* Bt,
                 bool b_c128, bool conj_b, int64_t ldb, int64_t sB, float2* C, int64_t ldc,
                 int64_t sC, int64_t M, int64_t N, int64_t K, int64_t batch, cudaStream_t s) {
  CQ_REQUIRE(M > 0 && N > 0 && K > 0 && batch > 0, COQUI_B200_EINVAL, "tc_cgemm: empty problem");
  TcParams p;
  p.A = A;
  p.Bt = Bt;
  p.C = C;
  p.M = M;
  p.N = N;
  p.K = K;
  p.lda = lda;
  p.ldb = ldb;
  p.ldc = ldc;
  p.sA = sA;
  p.sB = sB;
  p.sC = sC;
  p.a64 = a_c128;
  p.b64 = b_c128;
  p.conj_a = conj_a;
  p.conj_b = conj_b;
  if (a_c128 && b_c128) dispatch_n<true, true>(p, batch, s);
  else if (a_c128) dispatch_n<true, false>(p, batch, s);
  else if (b_c128) dispatch_n<false, true>(p, batch, s);
  else dispatch_n<false, false>(p, batch, s);
}

int tc_take_error() {
  int h = 0, z = 0;
  CQ_CHECK_CUDA(cudaMemcpyFromSymbol(&h, g_tc_error, sizeof(int)));
  if (h) CQ_CHECK_CUDA(cudaMemcpyToSymbol(g_tc_error, &z, sizeof(int)));
  return h;
}

// ---------------------------------------------------------------------------------------
// projections
// ---------------------------------------------------------------------------------------
__global__ void k_transpose_X(const double2* __restrict__ X, double2* __restrict__ XT, int64_t Np,
                              int64_t nb, int64_t nk) {
  const int64_t total = nk * Np * nb;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = i / (Np * nb), e = i % (Np * nb);
    const int64_t P = e / nb, a = e % nb;
    XT[k * Np * nb + a * Np + P] = X[i];
  }
}

void tc_pack_X(TcOperand& op, const double2* X, int64_t nk, int64_t Np, int64_t nb,
               cudaStream_t s) {
  op.X = X;
  op.nk = nk;
  op.Np = Np;
  op.nb = nb;
  op.packed.ensure((size_t)nk * Np * nb * sizeof(double2));
  k_transpose_X<<<grid_for(nk * Np * nb, 256), 256, 0, s>>>(X, (double2*)op.packed.p, Np, nb, nk);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void tc_project_p2a(TcOperand& op, const double2* Gk, float2* out, int64_t nk, int64_t Np,
                    int64_t nb, cudaStream_t s) {
  op.tmp.ensure((size_t)nk * Np * nb * sizeof(float2));
  float2* T = (float2*)op.tmp.p;
  // T = X G  (Np x nb, K = nb) on CUDA cores (small)
  GemmDesc d{};
  d.M = Np; d.N = nb; d.K = nb;
  d.sam = nb; d.sak = 1; d.sbk = nb; d.sbn = 1;
  d.scm = nb; d.scn = 1;
  d.batch = nk; d.bsa = Np * nb; d.bsb = nb * nb; d.bsc = Np * nb;
  d.alpha = make_double2(1, 0); d.beta = make_double2(0, 0);
  launch_gemm_simt<double2, double2, float2, float>(d, op.X, Gk, T, s);
  // out = T X^H: B(k=b, n=Q) = conj(X[Q][b]) -> Bt = X with conjugation (tensor cores)
  tc_cgemm_nt(T, false, false, nb, Np * nb, op.X, true, true, nb, Np * nb, out, Np, Np * Np, Np,
              Np, nb, nk, s);
}

void tc_project_a2p(TcOperand& op, const float2* Sk, double2* out, int64_t nk, int64_t Np,
                    int64_t nb, cudaStream_t s) {
  op.tmp.ensure((size_t)nk * Np * nb * sizeof(float2));
  float2* U = (float2*)op.tmp.p;
  // U = S X  (Np x nb, K = Np): Bt = X^T (nb x Np), tensor cores
  tc_cgemm_nt(Sk, false, false, Np, Np * Np, op.packed.p, true, false, Np, Np * nb, U, nb,
              Np * nb, Np, nb, Np, nk, s);
  // out = X^H U  (nb x nb, K = Np) on CUDA cores (small)
  GemmDesc e{};
  e.M = nb; e.N = nb; e.K = Np;
  e.sam = 1; e.sak = nb; e.conj_a = true;  // A(a, P) = conj(X[P][a])
  e.sbk = nb; e.sbn = 1;
  e.scm = nb; e.scn = 1;
  e.batch = nk; e.bsa = Np * nb; e.bsb = Np * nb; e.bsc = nb * nb;
  e.alpha = make_double2(1, 0); e.beta = make_double2(0, 0);
  launch_gemm_simt<double2, float2, double2, double>(e, op.X, U, out, s);
}

}  // namespace cq
