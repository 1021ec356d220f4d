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
// of K per pipeline stage = one 128-byte swizzle row.  Warps 0-7 stage operands (global ->
// registers, two stages ahead -> split -> swizzled st.shared) and then drain TMEM through a
// shared-memory transpose into coalesced rows; warp 8 allocates TMEM and one of its lanes
// issues the MMAs.  Known triangular structure of A or B trims each tile's K range.  Waits
// are bounded by a 2 s global-timer budget that sets an error flag instead of hanging.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>

#include "kernels.cuh"
#include "tc_gemm.cuh"

namespace cq {

namespace {

__device__ int g_tc_error = 0;
// set when an input of the primary -> auxiliary projection holds NaN or Inf (the split-TF32
// products do not carry non-finite values through reliably, so they are caught on the way in)
__device__ int g_nonfinite = 0;
// time limit of every bounded wait (ns); 2 s unless a test shortens it
constexpr unsigned long long kDefaultWaitNs = 2000000000ull;
__device__ unsigned long long g_tc_wait_ns = kDefaultWaitNs;

// Whether every row of an operand starts 16-byte aligned at even K: a complex64 operand needs
// an aligned base and even row and batch strides; pre-split values are 16 bytes each.
int rows_aligned(const void* X, bool split, int64_t ld, int64_t sX) {
  if ((reinterpret_cast<uintptr_t>(X) & 15) != 0) return 0;
  return split ? 1 : (ld % 2 == 0 && sX % 2 == 0);
}

constexpr int kBM = 128;
constexpr int kBKR = 32;  // real K per stage (128 bytes of fp32)
// tcgen05.alloc takes a power of two of at least 32 columns
constexpr int pow2_at_least(int x) { return x <= 32 ? 32 : 2 * pow2_at_least((x + 1) / 2); }
// BNC complex columns per tile (32, 64, 96 or 128); NP producer threads (warps 0..NP/32-1 stage operands, then
// drain the accumulator; warp NP/32 allocates TMEM and issues MMAs); ST pipeline stages.
// Long-K products use (NP = 256, ST = 2); short-K ones (K <= 64) use (NP = 128, ST = 1), whose
// smaller footprint lets several CTAs share an SM so one tile's epilogue overlaps another's
// main loop.
template <int BNC, int NP, int ST> struct TileCfg {
  static constexpr int BNC_ = BNC;                     // complex columns per tile
  static constexpr int NR = 2 * BNC;                   // UMMA N (real columns)
  static constexpr int NPROD = NP;
  static constexpr int NPW = NP / 32;
  static constexpr int STAGES = ST;
  static constexpr int THREADS = NP + 32;
  static constexpr int A_PLANE = kBM * 128;            // bytes of one A plane
  static constexpr int B_PLANE = NR * 128;             // bytes of one B plane
  static constexpr int STAGE = 2 * A_PLANE + 2 * B_PLANE;
  static constexpr int SMEM = ST * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  static constexpr int TMEM_COLS = pow2_at_least(NR);  // 64, 128 or 256 (192 -> 256)
  static constexpr int A_CHUNKS = kBM * 8 / NP;        // A chunks per producer thread
  static constexpr int B_CHUNKS = BNC * 8 / NP;        // B chunks per producer thread
  // kind::tf32 dense, F32 accumulate, K-major A and B, M = 128, N = NR
  static constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) |
                                    ((uint32_t)(NR >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
  // epilogue: each warp drains NR / 2 columns at a time through a 32 x (NR / 2 + 4) buffer
  static constexpr int HALVES = 8 / NPW;
  static constexpr int EPI_PITCH = NR / 2 + 4;
  static_assert(NPW * 32 * EPI_PITCH * 4 <= ST * STAGE, "epilogue buffer");
  static_assert(B_CHUNKS >= 1, "tile too narrow for the producer count");
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
  int a_upper, a_lower, b_lower, b_upper, lower_only;
  int upper_zero;        // tiles strictly below the diagonal: zeros, no products
  int a_ident, b_ident;  // operand + identity (complex64 operands only)
  // every row of the operand starts 16-byte aligned at even K (vector loads allowed)
  int a_al, b_al;
  // periodic batch index (0 = off): operand batch = (q0 + b) % mod, for per-q operands
  int64_t a_mod, a_q0, b_mod, b_q0;
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

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// try_wait that suspends the thread for at most hint_ns before reporting an incomplete phase
__device__ __forceinline__ bool mbar_try_hint(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t done;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
      : "=r"(done)
      : "r"(bar), "r"(parity), "r"(hint_ns)
      : "memory");
  return done != 0;
}

// Bounded wait for the phase with the given parity; returns false (and flags) on timeout.
// With the default limit the clock is read only after a first failed attempt and then every
// 16 attempts; a shorter limit also bounds each attempt's suspension and is checked after
// every attempt.
__device__ __forceinline__ bool mbar_wait_for(uint32_t bar, uint32_t parity, uint64_t limit) {
  if (limit >= kDefaultWaitNs) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 1;; ++i) {
      if (mbar_try(bar, parity)) return true;
      if ((i & 15u) == 0 && global_ns() - t0 > limit) {
        atomicExch(&g_tc_error, 1);
        return false;
      }
    }
  }
  const uint32_t hint = (uint32_t)(limit < 1000000ull ? (limit > 0 ? limit : 1) : 1000000ull);
  if (mbar_try_hint(bar, parity, hint)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    if (mbar_try_hint(bar, parity, hint)) return true;
    if (global_ns() - t0 > limit) {
      atomicExch(&g_tc_error, 1);
      return false;
    }
  }
}
// the pipeline's waits: the current limit (g_tc_wait_ns)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, g_tc_wait_ns);
}
// the wait for issued tensor-core work to retire before tensor memory is released: always the
// default limit, also when a test has shortened the pipeline's
__device__ __forceinline__ bool mbar_drain(uint32_t bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, kDefaultWaitNs);
}

// Rounds to TF32 (10 explicit mantissa bits), to nearest with ties away from zero, as integer
// arithmetic on the magnitude bits (two ALU operations, no conversion unit): a finite input
// gives its TF32 value with the low 13 bits cleared.
__device__ __forceinline__ uint32_t to_tf32(float x) {
  return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
}

// split x into TF32 hi + lo (hi = rna(x), lo = rna(x - hi))
__device__ __forceinline__ void split2(double x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32((float)x);
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

// Two consecutive complex values (k, k+1) of one operand row, as loaded from global.
template <bool C128> struct Pair;
template <> struct Pair<false> {
  float4 v;
  static constexpr int kBytes = 8;  // per complex value
  // both values inside K and the address 16-byte aligned
  __device__ __forceinline__ void load_fast(const unsigned char* p, bool row_ok) {
    v = row_ok ? __ldg(reinterpret_cast<const float4*>(p)) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __device__ __forceinline__ void load_edge(const unsigned char* base, int64_t k, int64_t kmax,
                                            bool row_ok) {
    const float2* p = reinterpret_cast<const float2*>(base);
    float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
    if (row_ok && k < kmax) a = __ldg(p);
    if (row_ok && k + 1 < kmax) b = __ldg(p + 1);
    v = make_float4(a.x, a.y, b.x, b.y);
  }
  __device__ __forceinline__ void get(float (&x)[4]) const {
    x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
  }
  // adds 1 to the real part of the first (e = 0) or second (e = 1) value
  __device__ __forceinline__ void add_one(int e) {
    if (e == 0) v.x += 1.f;
    else v.z += 1.f;
  }
};
// Pre-split operand: one float4 (hi.re, hi.im, lo.re, lo.im) per complex value, hi/lo TF32.
template <> struct Pair<true> {
  float4 a, b;
  static constexpr int kBytes = 16;  // per complex value
  __device__ __forceinline__ void load_fast(const unsigned char* base, bool row_ok) {
    const float4* p = reinterpret_cast<const float4*>(base);
    a = make_float4(0.f, 0.f, 0.f, 0.f);
    b = a;
    if (row_ok) {
      a = __ldg(p);
      b = __ldg(p + 1);
    }
  }
  __device__ __forceinline__ void load_edge(const unsigned char* base, int64_t k, int64_t kmax,
                                            bool row_ok) {
    const float4* p = reinterpret_cast<const float4*>(base);
    a = make_float4(0.f, 0.f, 0.f, 0.f);
    b = a;
    if (row_ok && k < kmax) a = __ldg(p);
    if (row_ok && k + 1 < kmax) b = __ldg(p + 1);
  }
  __device__ __forceinline__ void add_one(int) {}  // not used: rejected on the host
};

// The operand rows one producer thread stages, fixed for a tile: chunk j of the thread lies
// in row row0 + j * (producer threads / 8) at complex column 2 * (thread % 8) of the K block.
struct OpRows {
  const unsigned char* base;  // chunk 0 at k = 0
  int64_t step;               // bytes from one chunk's row to the next chunk's
  int64_t row0;               // operand row of chunk 0
  uint32_t ok;                // bit j: chunk j's row lies inside the operand
};

template <int NCH, int NP>
__device__ __forceinline__ OpRows op_rows(const void* X, int64_t ld, int64_t sX, int64_t bidx,
                                          int64_t rows, int64_t r0, int es) {
  OpRows o;
  const int t = threadIdx.x;
  o.row0 = r0 + (t >> 3);
  o.step = (int64_t)(NP / 8) * ld * es;
  o.base = reinterpret_cast<const unsigned char*>(X) + (bidx * sX + o.row0 * ld + 2 * (t & 7)) * es;
  o.ok = 0;
#pragma unroll
  for (int j = 0; j < NCH; ++j)
    if (o.row0 + j * (NP / 8) < rows) o.ok |= 1u << j;
  return o;
}

template <class Cfg, bool A64, bool B64> struct Staging {
  Pair<A64> a[Cfg::A_CHUNKS];
  Pair<B64> b[Cfg::B_CHUNKS];
  static constexpr int RSTEP = Cfg::NPROD / 8;  // rows between a thread's chunks

  // the K block of 16 complex columns starting at k0c
  __device__ __forceinline__ void load(const TcParams& p, const OpRows& ra, const OpRows& rb,
                                       int64_t k0c) {
    const int64_t k = k0c + 2 * (threadIdx.x & 7);
    const bool inner = k0c + 16 <= p.K;  // uniform over the CTA
    const int64_t offa = k0c * Pair<A64>::kBytes, offb = k0c * Pair<B64>::kBytes;
    if (inner && p.a_al) {
#pragma unroll
      for (int j = 0; j < Cfg::A_CHUNKS; ++j)
        a[j].load_fast(ra.base + j * ra.step + offa, (ra.ok >> j) & 1u);
    } else {
#pragma unroll
      for (int j = 0; j < Cfg::A_CHUNKS; ++j)
        a[j].load_edge(ra.base + j * ra.step + offa, k, p.K, (ra.ok >> j) & 1u);
    }
    if (p.a_ident) {
#pragma unroll
      for (int j = 0; j < Cfg::A_CHUNKS; ++j) {
        const int64_t m = ra.row0 + j * RSTEP;
        if (!((ra.ok >> j) & 1u)) continue;
        if (m == k && k < p.K) a[j].add_one(0);
        if (m == k + 1 && k + 1 < p.K) a[j].add_one(1);
      }
    }
    if (inner && p.b_al) {
#pragma unroll
      for (int j = 0; j < Cfg::B_CHUNKS; ++j)
        b[j].load_fast(rb.base + j * rb.step + offb, (rb.ok >> j) & 1u);
    } else {
#pragma unroll
      for (int j = 0; j < Cfg::B_CHUNKS; ++j)
        b[j].load_edge(rb.base + j * rb.step + offb, k, p.K, (rb.ok >> j) & 1u);
    }
    if (p.b_ident) {
#pragma unroll
      for (int j = 0; j < Cfg::B_CHUNKS; ++j) {
        const int64_t n = rb.row0 + j * RSTEP;
        if (!((rb.ok >> j) & 1u)) continue;
        if (n == k && k < p.K) b[j].add_one(0);
        if (n == k + 1 && k + 1 < p.K) b[j].add_one(1);
      }
    }
  }

  // hi/lo TF32 words of the two complex values of a chunk: (re0, im0, re1, im1); sgn is the
  // sign bit applied to the imaginary parts (conjugation)
  template <bool SPLIT>
  __device__ __forceinline__ static void words(const Pair<SPLIT>& q, uint32_t sgn, uint32_t (&h)[4],
                                               uint32_t (&l)[4]) {
    if constexpr (SPLIT) {
      h[0] = __float_as_uint(q.a.x); h[1] = __float_as_uint(q.a.y) ^ sgn;
      h[2] = __float_as_uint(q.b.x); h[3] = __float_as_uint(q.b.y) ^ sgn;
      l[0] = __float_as_uint(q.a.z); l[1] = __float_as_uint(q.a.w) ^ sgn;
      l[2] = __float_as_uint(q.b.z); l[3] = __float_as_uint(q.b.w) ^ sgn;
    } else {
      float v[4];
      q.get(v);
      v[1] = __uint_as_float(__float_as_uint(v[1]) ^ sgn);
      v[3] = __uint_as_float(__float_as_uint(v[3]) ^ sgn);
#pragma unroll
      for (int j = 0; j < 4; ++j) split2(v[j], h[j], l[j]);
    }
  }

  __device__ __forceinline__ void store(const TcParams& p, uint32_t sA_hi, uint32_t sA_lo,
                                        uint32_t sB_hi, uint32_t sB_lo) const {
    const int t = threadIdx.x;
    constexpr uint32_t SGN = 0x80000000u;
    const uint32_t ca = p.conj_a ? SGN : 0u, cb = p.conj_b ? SGN : 0u;
#pragma unroll
    for (int j = 0; j < Cfg::A_CHUNKS; ++j) {
      const int i = t + j * Cfg::NPROD;
      const int r = i >> 3, c = i & 7;
      uint32_t h[4], l[4];
      words<A64>(a[j], ca, h, l);
      const uint32_t off = sw128(r, c);
      st_shared_v4(sA_hi + off, h[0], h[1], h[2], h[3]);
      st_shared_v4(sA_lo + off, l[0], l[1], l[2], l[3]);
    }
#pragma unroll
    for (int j = 0; j < Cfg::B_CHUNKS; ++j) {
      const int i = t + j * Cfg::NPROD;
      const int r = i >> 3, c = i & 7;
      uint32_t h[4], l[4];  // (br0, bi0, br1, bi1) after conjugation
      words<B64>(b[j], cb, h, l);
      // realified rows: 2r = (br, -bi) pairs, 2r+1 = (bi, br) pairs
      const uint32_t o0 = sw128(2 * r, c), o1 = sw128(2 * r + 1, c);
      st_shared_v4(sB_hi + o0, h[0], h[1] ^ SGN, h[2], h[3] ^ SGN);
      st_shared_v4(sB_lo + o0, l[0], l[1] ^ SGN, l[2], l[3] ^ SGN);
      st_shared_v4(sB_hi + o1, h[1], h[0], h[3], h[2]);
      st_shared_v4(sB_lo + o1, l[1], l[0], l[3], l[2]);
    }
  }
};

// One output tile (rows m0.., columns n0.. of problem bz) of the split-TF32 product.
template <int BNC, int NP, int ST, bool A64, bool B64>
__device__ __forceinline__ void tc_tile(const TcParams& p, int64_t bz, int64_t m0, int64_t n0,
                                        unsigned char* smem_raw) {
  using Cfg = TileCfg<BNC, NP, ST>;
  constexpr int kStages = ST;
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * Cfg::STAGE);
  // bars[0..ST) full, bars[ST..2ST) empty, bars[2ST] accumulator ready, bars[2ST + 1] all
  // issued MMAs retired, then the TMEM base
  uint64_t* acc_bar = bars + 2 * kStages;
  uint64_t* done_bar = acc_bar + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (p.lower_only && n0 > m0 + kBM - 1) return;  // tile strictly above the diagonal

  // K blocks (16 complex each) that can be nonzero for this tile
  int kb_lo = 0, kb_hi = (int)((p.K + 15) / 16);
  if (p.a_upper) kb_lo = max(kb_lo, (int)(m0 / 16));
  if (p.b_lower) kb_lo = max(kb_lo, (int)(n0 / 16));
  if (p.a_lower) kb_hi = min(kb_hi, (int)((m0 + kBM - 1) / 16) + 1);
  if (p.b_upper) kb_hi = min(kb_hi, (int)((n0 + BNC - 1) / 16) + 1);
  if (p.upper_zero && m0 > n0 + BNC - 1) kb_hi = kb_lo;  // written as zeros
  const int nkb = max(kb_hi - kb_lo, 0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&bars[s]), Cfg::NPW);  // one arrival per producer warp
      mbar_init(smem_u32(&bars[kStages + s]), 1);
    }
    mbar_init(smem_u32(acc_bar), 1);
    mbar_init(smem_u32(done_bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == Cfg::NPW) {
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
  if (warp < Cfg::NPW) {
    // ---------------- producers: register prefetch ----------------
    // Long K (eight producer warps): two register sets alternate, so a K block's global
    // loads have two stage times to arrive before its split values go to shared memory.
    // Short K (four producer warps, twice the values per thread): one set, one stage ahead.
    constexpr int kAhead = (NP == 256) ? 2 : 1;
    const int64_t ba = p.a_mod ? (p.a_q0 + bz) % p.a_mod : bz;
    const int64_t bb = p.b_mod ? (p.b_q0 + bz) % p.b_mod : bz;
    const OpRows ra = op_rows<Cfg::A_CHUNKS, NP>(p.A, p.lda, p.sA, ba, p.M, m0, Pair<A64>::kBytes);
    const OpRows rb = op_rows<Cfg::B_CHUNKS, NP>(p.Bt, p.ldb, p.sB, bb, p.N, n0, Pair<B64>::kBytes);
    auto step = [&](Staging<Cfg, A64, B64>& st, int it) -> bool {
      const int s = it % kStages;
      const uint32_t ph = (uint32_t)(it / kStages) & 1u;
      if (!mbar_wait(smem_u32(&bars[kStages + s]), ph ^ 1u)) return false;
      unsigned char* sp = smem + s * Cfg::STAGE;
      const uint32_t a_hi = smem_u32(sp), a_lo = a_hi + Cfg::A_PLANE;
      const uint32_t b_hi = a_lo + Cfg::A_PLANE, b_lo = b_hi + Cfg::B_PLANE;
      st.store(p, a_hi, a_lo, b_hi, b_lo);
      // each thread's stores become visible to the tensor core (async proxy); the warp's
      // lanes are ordered by the warp barrier and one lane arrives for the warp
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bars[s]));
      if (it + kAhead < nkb) st.load(p, ra, rb, (int64_t)(kb_lo + it + kAhead) * 16);
      return true;
    };
    if constexpr (kAhead == 2) {
      Staging<Cfg, A64, B64> st0, st1;
      if (nkb > 0) st0.load(p, ra, rb, (int64_t)kb_lo * 16);
      if (nkb > 1) st1.load(p, ra, rb, (int64_t)(kb_lo + 1) * 16);
      for (int it = 0; it < nkb; it += 2) {
        if (!step(st0, it)) { ok = false; break; }
        if (it + 1 < nkb && !step(st1, it + 1)) { ok = false; break; }
      }
    } else {
      Staging<Cfg, A64, B64> st0;
      if (nkb > 0) st0.load(p, ra, rb, (int64_t)kb_lo * 16);
      for (int it = 0; it < nkb; ++it)
        if (!step(st0, it)) { ok = false; break; }
    }
    // ---------------- epilogue: TMEM -> registers -> smem -> coalesced rows ----------------
    const int q = warp & 3;  // TMEM lane quadrant
    float* buf = reinterpret_cast<float*>(smem) + warp * 32 * Cfg::EPI_PITCH;
    bool have = false;
    if (ok && nkb > 0) {
      have = mbar_wait(smem_u32(acc_bar), 0u);
      if (have) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    // all producers must be past their last smem stage before it is reused
    asm volatile("bar.sync 1, %0;" ::"r"(Cfg::NPROD) : "memory");
#pragma unroll 1
    for (int hp = 0; hp < Cfg::HALVES; ++hp) {
      const int h = (warp >> 2) * Cfg::HALVES + hp;  // column half
      const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(h * (Cfg::NR / 2));
#pragma unroll 1
      for (int j = 0; j < Cfg::NR / 64; ++j) {
        uint32_t v[32];
        if (have) {
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
        } else {
#pragma unroll
          for (int x = 0; x < 32; ++x) v[x] = 0u;
        }
        float4* dst = reinterpret_cast<float4*>(buf + lane * Cfg::EPI_PITCH + j * 32);
#pragma unroll
        for (int x = 0; x < 8; ++x)
          dst[x] = make_float4(__uint_as_float(v[4 * x]), __uint_as_float(v[4 * x + 1]),
                               __uint_as_float(v[4 * x + 2]), __uint_as_float(v[4 * x + 3]));
      }
      __syncwarp();
      // warp writes its 32 rows; each row half is BNC/2 complex = BNC floats
      const int64_t nh = n0 + h * (BNC / 2);
      for (int rr = 0; rr < 32; ++rr) {
        const int64_t m = m0 + q * 32 + rr;
        if (m >= p.M) break;
        float2* crow = p.C + bz * p.sC + m * p.ldc + nh;
        const float* src = buf + rr * Cfg::EPI_PITCH;
        for (int x = lane * 4; x < BNC; x += 128) {
          const int64_t n = nh + x / 2;
          const float4 val = *reinterpret_cast<const float4*>(src + x);
          if (n + 1 < p.N && ((reinterpret_cast<uintptr_t>(crow + x / 2) & 15) == 0)) {
            *reinterpret_cast<float4*>(crow + x / 2) = val;
          } else {
            if (n < p.N) crow[x / 2] = make_float2(val.x, val.y);
            if (n + 1 < p.N) crow[x / 2 + 1] = make_float2(val.z, val.w);
          }
        }
      }
      __syncwarp();
    }
  } else if (lane == 0) {
    // ---------------- MMA issuer (one lane of the last warp) ----------------
    for (int it = 0; it < nkb; ++it) {
      const int s = it % kStages;
      const uint32_t ph = (uint32_t)(it / kStages) & 1u;
      if (!mbar_wait(smem_u32(&bars[s]), ph)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_hi = smem_u32(smem + s * Cfg::STAGE), a_lo = a_hi + Cfg::A_PLANE;
      const uint32_t b_hi = a_lo + Cfg::A_PLANE, b_lo = b_hi + Cfg::B_PLANE;
#pragma unroll
      for (int kk = 0; kk < kBKR / 8; ++kk) {
        const uint32_t o = (uint32_t)kk * 32;  // 8 tf32 = 32 bytes along K
        const uint64_t ah = make_desc(a_hi + o), al = make_desc(a_lo + o);
        const uint64_t bh = make_desc(b_hi + o), bl = make_desc(b_lo + o);
        const uint32_t acc = (it > 0 || kk > 0) ? 1u : 0u;
        mma_tf32(tmem, al, bh, Cfg::IDESC, acc);
        mma_tf32(tmem, ah, bl, Cfg::IDESC, 1u);
        mma_tf32(tmem, ah, bh, Cfg::IDESC, 1u);
      }
      mma_commit(smem_u32(&bars[kStages + s]));  // frees the stage once these MMAs retire
    }
    if (ok && nkb > 0) mma_commit(smem_u32(acc_bar));
    // every issued MMA has retired before TMEM is released, also when a wait gave up
    mma_commit(smem_u32(done_bar));
    mbar_drain(smem_u32(done_bar), 0u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == Cfg::NPW) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)Cfg::TMEM_COLS)
                 : "memory");
  }
}

template <int BNC, int NP, int ST, bool A64, bool B64>
__global__ void __launch_bounds__(NP + 32, (NP == 128 ? 2 : 1))
    k_tc_cgemm(const __grid_constant__ TcParams p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  tc_tile<BNC, NP, ST, A64, B64>(p, blockIdx.z, (int64_t)blockIdx.y * kBM, (int64_t)blockIdx.x * BNC,
                                 smem_raw);
}

// Grouped form: one launch over several problems of different shapes and strides (each group
// a batched product); the flattened tile index picks the group by binary search.
struct TcGroupDev {
  TcParams p;
  int64_t tiles_n, tiles_m, tile_begin;
};

template <int BNC, int NP, int ST, bool A64, bool B64>
__global__ void __launch_bounds__(NP + 32, (NP == 128 ? 2 : 1))
    k_tc_cgemm_grouped(const TcGroupDev* __restrict__ groups, int ngroups) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ TcParams sp;
  __shared__ int64_t s_bz, s_m0, s_n0;
  if (threadIdx.x == 0) {
    const int64_t t = blockIdx.x;
    int lo = 0, hi = ngroups - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (groups[mid].tile_begin <= t) lo = mid;
      else hi = mid - 1;
    }
    const TcGroupDev& g = groups[lo];
    const int64_t local = t - g.tile_begin, per_b = g.tiles_n * g.tiles_m;
    const int64_t r = local % per_b;
    sp = g.p;
    s_bz = local / per_b;
    s_m0 = (r / g.tiles_n) * kBM;
    s_n0 = (r % g.tiles_n) * BNC;
  }
  __syncthreads();
  tc_tile<BNC, NP, ST, A64, B64>(sp, s_bz, s_m0, s_n0, smem_raw);
}

// ---------------------------------------------------------------------------------------
// Persistent form: one CTA per SM slot walks the tiles blockIdx.x, + gridDim.x, ... of the
// whole batch.  The producer warps stage K blocks across tile boundaries (the next tile's
// first blocks are loaded while this tile's last ones are stored), one lane issues the MMAs
// into one of two TMEM accumulators, and four epilogue warps drain the other accumulator
// (TMEM -> registers -> a 32 x 32 shared transpose per warp -> coalesced rows) while the next
// tile accumulates.  Each element is formed from the same products in the same K order as in
// k_tc_cgemm, so the results are identical.
// ---------------------------------------------------------------------------------------
template <int BNC, int NP, int ST> struct PCfg {
  using Base = TileCfg<BNC, NP, ST>;
  static constexpr int NPW = NP / 32;
  static constexpr int MMA_WARP = NPW;
  static constexpr int EPI_WARP0 = NPW + 1;  // four warps; TMEM lane quadrant = warp % 4
  static constexpr int THREADS = NP + 32 + 128;
  static constexpr int EPI_PITCH = 36;       // floats per row of a warp's 32 x 32 buffer
  static constexpr int EPI_BYTES = 4 * 32 * EPI_PITCH * 4;
  static constexpr int ACC_STRIDE = pow2_at_least(Base::NR);  // columns between accumulators
  static constexpr int TMEM_COLS = 2 * ACC_STRIDE;              // two accumulators
  static constexpr int SMEM_USED = ST * Base::STAGE + EPI_BYTES + 1024 /*align*/ + 256 /*barriers*/;
  // at least 120 KB, so that one CTA occupies an SM (two CTAs' TMEM accumulators could exceed
  // the SM's 512 columns, and a CTA waiting in tcgen05.alloc for a persistent neighbour would
  // wait for good)
  static constexpr int SMEM = SMEM_USED > 120 * 1024 ? SMEM_USED : 120 * 1024;
  // registers per thread: the whole register file for one CTA per SM.  Each of the four SM
  // sub-partitions holds 16384 registers for its share of the warps (allocated 256 per warp).
  static constexpr int WARPS_PER_SUB = (THREADS / 32 + 3) / 4;
  static constexpr int MAXREG_RAW = (16384 / (WARPS_PER_SUB * 256)) * 8;
  static constexpr int MAXREG = MAXREG_RAW > 255 ? 255 : MAXREG_RAW;
};

// K blocks (16 complex each) of one tile that can be nonzero, and whether the tile is
// written at all (lower_only tiles strictly above the diagonal are not)
struct TileK {
  int kb_lo, nkb;
  bool live;
};
__device__ __forceinline__ TileK tile_k(const TcParams& p, int64_t m0, int64_t n0, int bnc) {
  TileK t;
  t.live = !(p.lower_only && n0 > m0 + kBM - 1);
  int kb_lo = 0, kb_hi = (int)((p.K + 15) / 16);
  if (p.a_upper) kb_lo = max(kb_lo, (int)(m0 / 16));
  if (p.b_lower) kb_lo = max(kb_lo, (int)(n0 / 16));
  if (p.a_lower) kb_hi = min(kb_hi, (int)((m0 + kBM - 1) / 16) + 1);
  if (p.b_upper) kb_hi = min(kb_hi, (int)((n0 + bnc - 1) / 16) + 1);
  if (p.upper_zero && m0 > n0 + bnc - 1) kb_hi = kb_lo;  // written as zeros
  t.kb_lo = kb_lo;
  t.nkb = max(kb_hi - kb_lo, 0);
  return t;
}

struct TileId {
  int64_t bz, m0, n0;
};
__device__ __forceinline__ TileId tile_id(int64_t t, int64_t tm, int64_t tn, int bnc) {
  const int64_t per = tm * tn, r = t % per;
  return TileId{t / per, (r / tn) * kBM, (r % tn) * bnc};
}

// Producer cursor over the (tile, K block) pairs of this CTA that have work.
template <class Cfg>
struct PCursor {
  int64_t t;      // tile index
  int k;          // K block within the tile (0 .. nkb - 1)
  bool valid;
  int kb_lo, nkb;
  OpRows ra, rb;
};

template <class Cfg, bool A64, bool B64>
__device__ __forceinline__ void pcursor_tile(const TcParams& p, PCursor<Cfg>& c, int64_t total,
                                             int64_t tm, int64_t tn) {
  // first tile >= c.t (in steps of gridDim.x) with live K blocks
  for (; c.t < total; c.t += gridDim.x) {
    const TileId id = tile_id(c.t, tm, tn, Cfg::BNC_);
    const TileK tk = tile_k(p, id.m0, id.n0, Cfg::BNC_);
    if (!tk.live || tk.nkb == 0) continue;
    const int64_t ba = p.a_mod ? (p.a_q0 + id.bz) % p.a_mod : id.bz;
    const int64_t bb = p.b_mod ? (p.b_q0 + id.bz) % p.b_mod : id.bz;
    c.kb_lo = tk.kb_lo;
    c.nkb = tk.nkb;
    c.k = 0;
    c.ra = op_rows<Cfg::A_CHUNKS, Cfg::NPROD>(p.A, p.lda, p.sA, ba, p.M, id.m0, Pair<A64>::kBytes);
    c.rb = op_rows<Cfg::B_CHUNKS, Cfg::NPROD>(p.Bt, p.ldb, p.sB, bb, p.N, id.n0, Pair<B64>::kBytes);
    c.valid = true;
    return;
  }
  c.valid = false;
}

template <class Cfg, bool A64, bool B64>
__device__ __forceinline__ void pcursor_next(const TcParams& p, PCursor<Cfg>& c, int64_t total,
                                             int64_t tm, int64_t tn) {
  if (++c.k < c.nkb) return;
  c.t += gridDim.x;
  pcursor_tile<Cfg, A64, B64>(p, c, total, tm, tn);
}

template <int BNC, int NP, int ST, bool A64, bool B64>
__global__ void __maxnreg__((PCfg<BNC, NP, ST>::MAXREG))
    k_tc_persistent(const __grid_constant__ TcParams p, int64_t batch) {
  using PC = PCfg<BNC, NP, ST>;
  using Cfg = TileCfg<BNC, NP, ST>;
  constexpr int kStages = ST;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  float* epi = reinterpret_cast<float*>(smem + kStages * Cfg::STAGE);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * Cfg::STAGE + PC::EPI_BYTES);
  // bars[0..ST) full, [ST..2ST) empty, acc_full[2], acc_empty[2], done, then the TMEM base
  uint64_t* acc_full = bars + 2 * kStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* done_bar = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t tm = (p.M + kBM - 1) / kBM, tn = (p.N + BNC - 1) / BNC;
  const int64_t total = tm * tn * batch;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&bars[s]), Cfg::NPW);
      mbar_init(smem_u32(&bars[kStages + s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&acc_full[b]), 1);
      mbar_init(smem_u32(&acc_empty[b]), 4);  // one arrival per epilogue warp
    }
    mbar_init(smem_u32(done_bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == PC::MMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"((uint32_t)PC::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp < Cfg::NPW) {
    // ---------------- producers ----------------
    constexpr int kAhead = (NP == 256) ? 2 : 1;
    PCursor<Cfg> L, S;
    L.t = blockIdx.x;
    pcursor_tile<Cfg, A64, B64>(p, L, total, tm, tn);
    S = L;
    int64_t g = 0;  // stage sequence number
    auto step = [&](Staging<Cfg, A64, B64>& st) -> bool {
      const int s = (int)(g % kStages);
      const uint32_t ph = (uint32_t)(g / kStages) & 1u;
      if (!mbar_wait(smem_u32(&bars[kStages + s]), ph ^ 1u)) return false;
      unsigned char* sp = smem + s * Cfg::STAGE;
      const uint32_t a_hi = smem_u32(sp), a_lo = a_hi + Cfg::A_PLANE;
      const uint32_t b_hi = a_lo + Cfg::A_PLANE, b_lo = b_hi + Cfg::B_PLANE;
      st.store(p, a_hi, a_lo, b_hi, b_lo);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bars[s]));
      if (L.valid) {
        st.load(p, L.ra, L.rb, (int64_t)(L.kb_lo + L.k) * 16);
        pcursor_next<Cfg, A64, B64>(p, L, total, tm, tn);
      }
      pcursor_next<Cfg, A64, B64>(p, S, total, tm, tn);
      ++g;
      return true;
    };
    if constexpr (kAhead == 2) {
      Staging<Cfg, A64, B64> st0, st1;
      if (L.valid) {
        st0.load(p, L.ra, L.rb, (int64_t)(L.kb_lo + L.k) * 16);
        pcursor_next<Cfg, A64, B64>(p, L, total, tm, tn);
      }
      if (L.valid) {
        st1.load(p, L.ra, L.rb, (int64_t)(L.kb_lo + L.k) * 16);
        pcursor_next<Cfg, A64, B64>(p, L, total, tm, tn);
      }
      while (S.valid) {
        if (!step(st0)) break;
        if (!S.valid || !step(st1)) break;
      }
    } else {
      Staging<Cfg, A64, B64> st0;
      if (L.valid) {
        st0.load(p, L.ra, L.rb, (int64_t)(L.kb_lo + L.k) * 16);
        pcursor_next<Cfg, A64, B64>(p, L, total, tm, tn);
      }
      while (S.valid)
        if (!step(st0)) break;
    }
  } else if (warp == PC::MMA_WARP) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int64_t g = 0, u = 0;  // stage sequence, accumulator uses
      bool ok = true;
      for (int64_t t = blockIdx.x; t < total && ok; t += gridDim.x) {
        const TileId id = tile_id(t, tm, tn, BNC);
        const TileK tk = tile_k(p, id.m0, id.n0, BNC);
        if (!tk.live || tk.nkb == 0) continue;
        const int b = (int)(u & 1);
        if (!mbar_wait(smem_u32(&acc_empty[b]), (uint32_t)((u >> 1) & 1) ^ 1u)) { ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc_t = tmem + (uint32_t)(b * PC::ACC_STRIDE);
        for (int it = 0; it < tk.nkb; ++it, ++g) {
          const int s = (int)(g % kStages);
          const uint32_t ph = (uint32_t)(g / kStages) & 1u;
          if (!mbar_wait(smem_u32(&bars[s]), ph)) { ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a_hi = smem_u32(smem + s * Cfg::STAGE), a_lo = a_hi + Cfg::A_PLANE;
          const uint32_t b_hi = a_lo + Cfg::A_PLANE, b_lo = b_hi + Cfg::B_PLANE;
#pragma unroll
          for (int kk = 0; kk < kBKR / 8; ++kk) {
            const uint32_t o = (uint32_t)kk * 32;
            const uint64_t ah = make_desc(a_hi + o), al = make_desc(a_lo + o);
            const uint64_t bh = make_desc(b_hi + o), bl = make_desc(b_lo + o);
            const uint32_t acc = (it > 0 || kk > 0) ? 1u : 0u;
            mma_tf32(acc_t, al, bh, Cfg::IDESC, acc);
            mma_tf32(acc_t, ah, bl, Cfg::IDESC, 1u);
            mma_tf32(acc_t, ah, bh, Cfg::IDESC, 1u);
          }
          mma_commit(smem_u32(&bars[kStages + s]));
        }
        if (!ok) break;
        mma_commit(smem_u32(&acc_full[b]));
        ++u;
      }
      // every MMA this lane issued has retired before TMEM is released
      mma_commit(smem_u32(done_bar));
      mbar_drain(smem_u32(done_bar), 0u);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue: TMEM -> registers -> smem -> coalesced rows ----------------
    const int q = warp & 3;  // TMEM lane quadrant
    float* buf = epi + (warp - PC::EPI_WARP0) * 32 * PC::EPI_PITCH;
    int64_t u = 0;
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
      const TileId id = tile_id(t, tm, tn, BNC);
      const TileK tk = tile_k(p, id.m0, id.n0, BNC);
      if (!tk.live) continue;
      const bool have = tk.nkb > 0;
      const int b = (int)(u & 1);
      if (have) {
        if (!mbar_wait(smem_u32(&acc_full[b]), (uint32_t)((u >> 1) & 1))) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      }
      const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * PC::ACC_STRIDE);
#pragma unroll 1
      for (int j = 0; j < Cfg::NR / 32; ++j) {
        uint32_t v[32];
        if (have) {
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
          if (j == Cfg::NR / 32 - 1) {
            // the accumulator is read out: the MMA lane may reuse it
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
          }
        } else {
#pragma unroll
          for (int x = 0; x < 32; ++x) v[x] = 0u;
        }
        float4* dst = reinterpret_cast<float4*>(buf + lane * PC::EPI_PITCH);
#pragma unroll
        for (int x = 0; x < 8; ++x)
          dst[x] = make_float4(__uint_as_float(v[4 * x]), __uint_as_float(v[4 * x + 1]),
                               __uint_as_float(v[4 * x + 2]), __uint_as_float(v[4 * x + 3]));
        __syncwarp();
        // 32 rows x 16 complex columns: lanes 8 r' .. 8 r' + 7 write one row (128 bytes)
        const int64_t nc = id.n0 + j * 16 + (lane & 7) * 2;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int rr = 4 * i + (lane >> 3);
          const int64_t m = id.m0 + q * 32 + rr;
          if (m >= p.M) continue;
          const float4 val = *reinterpret_cast<const float4*>(buf + rr * PC::EPI_PITCH + (lane & 7) * 4);
          float2* cp = p.C + id.bz * p.sC + m * p.ldc + nc;
          if (nc + 1 < p.N && ((reinterpret_cast<uintptr_t>(cp) & 15) == 0)) {
            *reinterpret_cast<float4*>(cp) = val;
          } else {
            if (nc < p.N) cp[0] = make_float2(val.x, val.y);
            if (nc + 1 < p.N) cp[1] = make_float2(val.z, val.w);
          }
        }
        __syncwarp();
      }
      if (have) ++u;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == PC::MMA_WARP) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)PC::TMEM_COLS)
                 : "memory");
  }
}

template <int BNC, int NP, int ST, bool A64, bool B64>
void launch_tc_persistent(const TcParams& p, int64_t batch, cudaStream_t s) {
  using PC = PCfg<BNC, NP, ST>;
  auto fn = k_tc_persistent<BNC, NP, ST, A64, B64>;
  static int slots[64] = {};
  int dev = 0;
  CQ_CHECK_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && slots[dev] == 0) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, PC::SMEM));
    int per_sm = 0, sms = 0;
    CQ_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PC::THREADS, PC::SMEM));
    CQ_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // co-resident CTAs must fit their TMEM accumulators (512 columns per SM): tcgen05.alloc of
    // a CTA would otherwise wait for another CTA that never exits
    CQ_REQUIRE(per_sm >= 1 && per_sm * PC::TMEM_COLS <= 512, COQUI_B200_ECUDA,
               "tc_cgemm: persistent tile configuration does not fit an SM (" +
                   std::to_string(per_sm) + " CTAs of " + std::to_string(PC::TMEM_COLS) +
                   " TMEM columns)");
    slots[dev] = sms * per_sm;
  }
  const int64_t tiles = ((p.M + kBM - 1) / kBM) * ((p.N + BNC - 1) / BNC) * batch;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(tiles, dev < 64 ? slots[dev] : 148));
  fn<<<(unsigned)grid, PC::THREADS, PC::SMEM, s>>>(p, batch);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

template <int BNC, int NP, int ST, bool A64, bool B64>
void launch_tc(const TcParams& p, int64_t batch, cudaStream_t s) {
  using Cfg = TileCfg<BNC, NP, ST>;
  auto fn = k_tc_cgemm<BNC, NP, ST, A64, B64>;
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
    if (p.a_mod)
      q.a_q0 = (p.a_q0 + b0) % p.a_mod;
    else
      q.A = (const unsigned char*)p.A + b0 * p.sA * (p.a64 ? 16 : 8);  // split = 16 B
    if (p.b_mod)
      q.b_q0 = (p.b_q0 + b0) % p.b_mod;
    else
      q.Bt = (const unsigned char*)p.Bt + b0 * p.sB * (p.b64 ? 16 : 8);
    q.C = p.C + b0 * p.sC;
    dim3 grid((unsigned)((p.N + BNC - 1) / BNC), (unsigned)((p.M + kBM - 1) / kBM), (unsigned)nb);
    fn<<<grid, Cfg::THREADS, Cfg::SMEM, s>>>(q);
    count_launch();
    CQ_CHECK_CUDA(cudaGetLastError());
  }
}

// Tile configurations: (BNC, producer threads, stages), 0-5 with one tile per CTA
// (k_tc_cgemm) and 6-11 the same tiles in the persistent kernel; 12-15 the 96-column tile
// (UMMA N = 192: products with N = nb = 96 in one column tile, each A block staged once) in
// both forms.  Every configuration forms the same products in the same K order, so the
// results are identical and only the speed differs.
constexpr int kNumCfg = 16;

template <bool A64, bool B64>
void launch_cfg(int cfg, const TcParams& p, int64_t batch, cudaStream_t s) {
  switch (cfg) {
    case 6: return launch_tc_persistent<32, 128, 1, A64, B64>(p, batch, s);
    case 7: return launch_tc_persistent<64, 128, 1, A64, B64>(p, batch, s);
    case 8: return launch_tc_persistent<128, 128, 1, A64, B64>(p, batch, s);
    case 9: return launch_tc_persistent<32, 256, 2, A64, B64>(p, batch, s);
    case 10: return launch_tc_persistent<64, 256, 2, A64, B64>(p, batch, s);
    case 11: return launch_tc_persistent<128, 256, 2, A64, B64>(p, batch, s);
    case 12: return launch_tc<96, 128, 1, A64, B64>(p, batch, s);
    case 13: return launch_tc<96, 256, 2, A64, B64>(p, batch, s);
    case 14: return launch_tc_persistent<96, 128, 1, A64, B64>(p, batch, s);
    case 15: return launch_tc_persistent<96, 256, 2, A64, B64>(p, batch, s);
    default: break;
  }
  switch (cfg) {
    case 0: launch_tc<32, 128, 1, A64, B64>(p, batch, s); break;
    case 1: launch_tc<64, 128, 1, A64, B64>(p, batch, s); break;
    case 2: launch_tc<128, 128, 1, A64, B64>(p, batch, s); break;
    case 3: launch_tc<32, 256, 2, A64, B64>(p, batch, s); break;
    case 4: launch_tc<64, 256, 2, A64, B64>(p, batch, s); break;
    default: launch_tc<128, 256, 2, A64, B64>(p, batch, s); break;
  }
}

// Default choice: short K gets one stage and four producer warps (several CTAs per SM), long
// K two stages and eight producer warps; the tile width follows N.
int heuristic_cfg(const TcParams& p) {
  if (p.N > 64 && p.N <= 96) return p.K <= 64 ? 12 : 13;  // one 96-column tile
  const int w = p.N >= 128 ? 2 : (p.N > 32 ? 1 : 0);
  return (p.K <= 64 ? 0 : 3) + w;
}

// Autotuner: the first product of each shape class runs every configuration once (timed with
// CUDA events on the launching stream) and the fastest is kept for the class.
std::atomic<int> g_autotune{-1};  // -1: not yet read from COQUI_B200_AUTOTUNE (default on)
std::mutex g_tune_mu;
std::map<std::vector<int64_t>, int> g_tuned;

bool autotune_on() {
  int v = g_autotune.load();
  if (v < 0) {
    const char* e = std::getenv("COQUI_B200_AUTOTUNE");
    v = (e && e[0] == '0') ? 0 : 1;
    g_autotune.store(v);
  }
  return v == 1;
}

std::atomic<int> g_forced_cfg{-1};

template <bool A64, bool B64>
void dispatch_n(const TcParams& p, int64_t batch, cudaStream_t s) {
  const int forced = g_forced_cfg.load();
  if (forced >= 0) return launch_cfg<A64, B64>(forced, p, batch, s);
  if (!autotune_on()) return launch_cfg<A64, B64>(heuristic_cfg(p), p, batch, s);
  int64_t bb = 1;
  while (bb < batch) bb <<= 1;  // batch class: next power of two
  const std::vector<int64_t> key = {p.M, p.N, p.K, bb, A64, B64, p.conj_a, p.conj_b, p.a_upper,
                                    p.a_lower, p.b_lower, p.b_upper, p.lower_only, p.upper_zero};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) return launch_cfg<A64, B64>(it->second, p, batch, s);
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CQ_CHECK_CUDA(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone) return launch_cfg<A64, B64>(heuristic_cfg(p), p, batch, s);
  cudaEvent_t ev[kNumCfg + 1];
  for (auto& e : ev) CQ_CHECK_CUDA(cudaEventCreate(&e));
  CQ_CHECK_CUDA(cudaEventRecord(ev[0], s));
  for (int c = 0; c < kNumCfg; ++c) {
    launch_cfg<A64, B64>(c, p, batch, s);
    CQ_CHECK_CUDA(cudaEventRecord(ev[c + 1], s));
  }
  CQ_CHECK_CUDA(cudaEventSynchronize(ev[kNumCfg]));
  int best = heuristic_cfg(p);
  float best_ms = 1e30f;
  for (int c = 0; c < kNumCfg; ++c) {
    float ms = 0;
    CQ_CHECK_CUDA(cudaEventElapsedTime(&ms, ev[c], ev[c + 1]));
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[key] = best;
}

}  // namespace

void tc_cgemm_nt(const void* A, bool a_split, bool conj_a, int64_t lda, int64_t sA, const void* Bt,
                 bool b_split, bool conj_b, int64_t ldb, int64_t sB, float2* C, int64_t ldc,
                 int64_t sC, int64_t M, int64_t N, int64_t K, int64_t batch, cudaStream_t s,
                 const TcStructure& st) {
  const bool a_c128 = a_split, b_c128 = b_split;
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
  p.a_upper = st.a_upper;
  p.a_lower = st.a_lower;
  p.b_lower = st.b_lower;
  p.b_upper = st.b_upper;
  p.lower_only = st.lower_only;
  p.upper_zero = st.upper_zero;
  CQ_REQUIRE(!(st.a_ident && a_c128) && !(st.b_ident && b_c128), COQUI_B200_EINVAL,
             "tc_cgemm: identity shift needs a complex64 operand");
  p.a_ident = st.a_ident;
  p.b_ident = st.b_ident;
  p.a_al = rows_aligned(A, a_c128, lda, sA);
  p.b_al = rows_aligned(Bt, b_c128, ldb, sB);
  p.a_mod = st.a_mod;
  p.a_q0 = st.a_q0;
  p.b_mod = st.b_mod;
  p.b_q0 = st.b_q0;
  if (a_c128 && b_c128) dispatch_n<true, true>(p, batch, s);
  else if (a_c128) dispatch_n<true, false>(p, batch, s);
  else if (b_c128) dispatch_n<false, true>(p, batch, s);
  else dispatch_n<false, false>(p, batch, s);
}

int tc_take_nonfinite() {
  int h = 0, z = 0;
  CQ_CHECK_CUDA(cudaMemcpyFromSymbol(&h, g_nonfinite, sizeof(int)));
  if (h) CQ_CHECK_CUDA(cudaMemcpyToSymbol(g_nonfinite, &z, sizeof(int)));
  return h;
}

void tc_set_wait_ns(int64_t ns) {
  const unsigned long long v = ns > 0 ? (unsigned long long)ns : kDefaultWaitNs;
  CQ_CHECK_CUDA(cudaMemcpyToSymbol(g_tc_wait_ns, &v, sizeof(v)));
}

int tc_take_error() {
  int h = 0, z = 0;
  CQ_CHECK_CUDA(cudaMemcpyFromSymbol(&h, g_tc_error, sizeof(int)));
  if (h) CQ_CHECK_CUDA(cudaMemcpyToSymbol(g_tc_error, &z, sizeof(int)));
  return h;
}

// ---------------------------------------------------------------------------------------
// operand preparation and projections
// ---------------------------------------------------------------------------------------
// out (float4 per complex: hi.re, hi.im, lo.re, lo.im) from complex128; if transpose, the
// (rows x cols) blocks are written transposed (cols x rows).
__global__ void k_to_split(const double2* __restrict__ in, float4* __restrict__ out, int64_t rows,
                           int64_t cols, int64_t total, int transpose) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 x = in[i];
    uint32_t hr, lr, hi, li;
    split2(x.x, hr, lr);
    split2(x.y, hi, li);
    int64_t o = i;
    if (transpose) {
      const int64_t b = i / (rows * cols), e = i % (rows * cols);
      o = b * rows * cols + (e % cols) * rows + e / cols;
    }
    out[o] = make_float4(__uint_as_float(hr), __uint_as_float(hi), __uint_as_float(lr),
                         __uint_as_float(li));
  }
}

// out = in as complex64; if transpose, the (rows x cols) blocks are written transposed
__global__ void k_to_c64(const double2* __restrict__ in, float2* __restrict__ out, int64_t rows,
                         int64_t cols, int64_t total, int transpose) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 x = in[i];
    int64_t o = i;
    if (transpose) {
      const int64_t b = i / (rows * cols), e = i % (rows * cols);
      o = b * rows * cols + (e % cols) * rows + e / cols;
    }
    out[o] = make_float2((float)x.x, (float)x.y);
  }
}

// out[b] = in[b]^T as complex64, (rows x cols) blocks of complex128
__global__ void k_transpose_c64(const double2* __restrict__ in, float2* __restrict__ out,
                                int64_t rows, int64_t cols, int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / (rows * cols), e = i % (rows * cols);
    const double2 x = in[i];
    if (!isfinite(x.x) || !isfinite(x.y)) atomicExch(&g_nonfinite, 1);
    out[b * rows * cols + (e % cols) * rows + e / cols] = make_float2((float)x.x, (float)x.y);
  }
}

// out[b] = in[b]^T, (rows x cols) complex64 blocks; 32 x 32 tiles through shared memory
__global__ void k_transpose_f2(const float2* __restrict__ in, float2* __restrict__ out,
                               int64_t rows, int64_t cols) {
  __shared__ float2 tile[32][33];
  const int64_t b = blockIdx.z;
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  const float2* src = in + b * rows * cols;
  float2* dst = out + b * rows * cols;
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    const int64_t r = r0 + ty, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[ty][threadIdx.x] = src[r * cols + c];
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    const int64_t c = c0 + ty, r = r0 + threadIdx.x;  // out row c, column r
    if (r < rows && c < cols) dst[c * rows + r] = tile[threadIdx.x][ty];
  }
}

__global__ void k_c64_to_c128(const float2* __restrict__ in, double2* __restrict__ out,
                              int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = make_double2(in[i].x, in[i].y);
}

void to_split(const double2* in, float4* out, int64_t rows, int64_t cols, int64_t batch,
              bool transpose, cudaStream_t s) {
  const int64_t total = rows * cols * batch;
  k_to_split<<<grid_for(total, 256), 256, 0, s>>>(in, out, rows, cols, total, transpose ? 1 : 0);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void to_c64(const double2* in, float2* out, int64_t rows, int64_t cols, int64_t batch,
            bool transpose, cudaStream_t s) {
  const int64_t total = rows * cols * batch;
  k_to_c64<<<grid_for(total, 256), 256, 0, s>>>(in, out, rows, cols, total, transpose ? 1 : 0);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void tc_pack_X(TcOperand& op, const double2* X, int64_t nk, int64_t Np, int64_t nb,
               cudaStream_t s) {
  op.X = X;
  op.nk = nk;
  op.Np = Np;
  op.nb = nb;
  op.packed.ensure((size_t)nk * Np * nb * sizeof(float2) * 2);
  float2* Xc = (float2*)op.packed.p;
  to_c64(X, Xc, Np, nb, nk, false, s);                 // X   (nk, Np, nb)
  to_c64(X, Xc + nk * Np * nb, Np, nb, nk, true, s);   // X^T (nk, nb, Np)
}

void tc_project_p2a(TcOperand& op, const double2* Gk, float2* out, int64_t nk, int64_t Np,
                    int64_t nb, int64_t nbatch, cudaStream_t s) {
  const float2* Xs = (const float2*)op.packed.p;
  op.tmp.ensure((size_t)nbatch * Np * nb * sizeof(float2) + (size_t)nbatch * nb * nb * sizeof(float2));
  float2* T = (float2*)op.tmp.p;
  float2* Gt = T + nbatch * Np * nb;
  const int64_t tg = nbatch * nb * nb;
  k_transpose_c64<<<grid_for(tg, 256), 256, 0, s>>>(Gk, Gt, nb, nb, tg);
  count_launch();
  // problem b = (tau, k) uses X^k: X is addressed periodically with period nk
  TcStructure sx_a, sx_b;
  sx_a.a_mod = nk;
  sx_b.b_mod = nk;
  // T = X G  (Np x nb, K = nb): Bt[j][i] = G[i][j]
  tc_cgemm_nt(Xs, false, false, nb, Np * nb, Gt, false, false, nb, nb * nb, T, nb, Np * nb, Np,
              nb, nb, nbatch, s, sx_a);
  // out = T X^H: B(k=b, n=Q) = conj(X[Q][b])
  tc_cgemm_nt(T, false, false, nb, Np * nb, Xs, false, true, nb, Np * nb, out, Np, Np * Np, Np,
              Np, nb, nbatch, s, sx_b);
}

void tc_project_a2p(TcOperand& op, const float2* Sk, double2* out, int64_t nk, int64_t Np,
                    int64_t nb, int64_t nbatch, cudaStream_t s) {
  const float2* XTs = (const float2*)op.packed.p + nk * Np * nb;
  op.tmp.ensure((size_t)nbatch * Np * nb * sizeof(float2) + (size_t)nbatch * nb * nb * sizeof(float2));
  float2* UT = (float2*)op.tmp.p;
  float2* Sab = UT + nbatch * Np * nb;
  // U = S X (Np x nb, K = Np) with the Np rows on the 128-row tiles, then U^T (the big product
  // would waste half of every tile with the nb rows of U^T = X^T S^T on them)
  op.tmp2.ensure((size_t)nbatch * Np * nb * sizeof(float2));
  float2* U = (float2*)op.tmp2.p;
  TcStructure sb;
  sb.b_mod = nk;
  tc_cgemm_nt(Sk, false, false, Np, Np * Np, XTs, false, false, Np, nb * Np, U, nb, Np * nb, Np,
              nb, Np, nbatch, s, sb);
  CQ_REQUIRE(nbatch <= 65535, COQUI_B200_EINVAL, "a2p: too many problems per launch");
  k_transpose_f2<<<dim3((unsigned)((nb + 31) / 32), (unsigned)((Np + 31) / 32), (unsigned)nbatch),
                   dim3(32, 8), 0, s>>>(U, UT, Np, nb);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  TcStructure sx;
  sx.a_mod = nk;
  // Sigma_ab = X^H U (nb x nb, K = Np): A(a, P) = conj(X^T[a][P]), Bt = U^T
  tc_cgemm_nt(XTs, false, true, Np, nb * Np, UT, false, false, Np, nb * Np, Sab, nb, nb * nb, nb,
              nb, Np, nbatch, s, sx);
  const int64_t t = nbatch * nb * nb;
  k_c64_to_c128<<<grid_for(t, 256), 256, 0, s>>>(Sab, out, t);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

namespace {
TcParams make_params(const TcGroup& g) {
  TcParams p;
  p.A = g.A;
  p.Bt = g.Bt;
  p.C = g.C;
  p.M = g.M;
  p.N = g.N;
  p.K = g.K;
  p.lda = g.lda;
  p.ldb = g.ldb;
  p.ldc = g.ldc;
  p.sA = g.sA;
  p.sB = g.sB;
  p.sC = g.sC;
  p.a64 = g.a_split;
  p.b64 = g.b_split;
  p.conj_a = g.conj_a;
  p.conj_b = g.conj_b;
  p.a_upper = g.st.a_upper;
  p.a_lower = g.st.a_lower;
  p.b_lower = g.st.b_lower;
  p.b_upper = g.st.b_upper;
  p.lower_only = g.st.lower_only;
  p.upper_zero = g.st.upper_zero;
  p.a_ident = g.st.a_ident;
  p.b_ident = g.st.b_ident;
  p.a_al = rows_aligned(g.A, g.a_split, g.lda, g.sA);
  p.b_al = rows_aligned(g.Bt, g.b_split, g.ldb, g.sB);
  p.a_mod = g.st.a_mod;
  p.a_q0 = g.st.a_q0;
  p.b_mod = g.st.b_mod;
  p.b_q0 = g.st.b_q0;
  return p;
}

template <int BNC, int NP, int ST, bool A64, bool B64>
void launch_grouped(const std::vector<TcGroup>& gs, DevBuf<unsigned char>& table, cudaStream_t s) {
  using Cfg = TileCfg<BNC, NP, ST>;
  auto fn = k_tc_cgemm_grouped<BNC, NP, ST, A64, B64>;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
    attr_set[dev] = true;
  }
  std::vector<TcGroupDev> h;
  int64_t tiles = 0;
  for (const TcGroup& g : gs) {
    TcGroupDev d;
    d.p = make_params(g);
    d.tiles_n = (g.N + BNC - 1) / BNC;
    d.tiles_m = (g.M + kBM - 1) / kBM;
    d.tile_begin = tiles;
    tiles += d.tiles_n * d.tiles_m * g.batch;
    h.push_back(d);
  }
  CQ_REQUIRE(tiles <= 2147483647, COQUI_B200_EINVAL, "tc_cgemm_grouped: too many tiles");
  table.ensure(h.size() * sizeof(TcGroupDev));
  CQ_CHECK_CUDA(cudaMemcpyAsync(table.p, h.data(), h.size() * sizeof(TcGroupDev),
                                cudaMemcpyHostToDevice, s));
  fn<<<(unsigned)tiles, Cfg::THREADS, Cfg::SMEM, s>>>((const TcGroupDev*)table.p, (int)h.size());
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

template <bool A64, bool B64>
void grouped_dispatch(const std::vector<TcGroup>& gs, DevBuf<unsigned char>& table, cudaStream_t s) {
  int64_t maxK = 0, maxN = 0;
  for (const TcGroup& g : gs) {
    maxK = std::max(maxK, g.K);
    maxN = std::max(maxN, g.N);
  }
  if (maxK <= 64) {
    if (maxN >= 128) launch_grouped<128, 128, 1, A64, B64>(gs, table, s);
    else if (maxN > 32) launch_grouped<64, 128, 1, A64, B64>(gs, table, s);
    else launch_grouped<32, 128, 1, A64, B64>(gs, table, s);
  } else {
    if (maxN >= 128) launch_grouped<128, 256, 2, A64, B64>(gs, table, s);
    else if (maxN > 32) launch_grouped<64, 256, 2, A64, B64>(gs, table, s);
    else launch_grouped<32, 256, 2, A64, B64>(gs, table, s);
  }
}
}  // namespace

void tc_cgemm_grouped(const std::vector<TcGroup>& groups, DevBuf<unsigned char>& table,
                      cudaStream_t s) {
  if (groups.empty()) return;
  const bool a64 = groups[0].a_split, b64 = groups[0].b_split;
  for (const TcGroup& g : groups) {
    CQ_REQUIRE(g.a_split == a64 && g.b_split == b64, COQUI_B200_EINVAL,
               "tc_cgemm_grouped: all groups need the same operand formats");
    CQ_REQUIRE(g.M > 0 && g.N > 0 && g.K > 0 && g.batch > 0, COQUI_B200_EINVAL,
               "tc_cgemm_grouped: empty group");
    CQ_REQUIRE(!(g.st.a_ident && g.a_split) && !(g.st.b_ident && g.b_split), COQUI_B200_EINVAL,
               "tc_cgemm_grouped: identity shift needs a complex64 operand");
  }
  // longest tiles first: CTAs start in tile order, so the groups with the longest K (the
  // largest problems) must not be left for the tail of the launch
  std::vector<TcGroup> order(groups);
  std::stable_sort(order.begin(), order.end(),
                   [](const TcGroup& x, const TcGroup& y) { return x.K > y.K; });
  if (a64 && b64) grouped_dispatch<true, true>(order, table, s);
  else if (a64) grouped_dispatch<true, false>(order, table, s);
  else if (b64) grouped_dispatch<false, true>(order, table, s);
  else grouped_dispatch<false, false>(order, table, s);
}

void tc_set_autotune(int on) { g_autotune.store(on ? 1 : 0); }

bool tc_set_forced_cfg(int cfg) {
  if (cfg < -1 || cfg >= kNumCfg) return false;
  g_forced_cfg.store(cfg);
  return true;
}

int tc_num_cfgs() { return kNumCfg; }

int64_t tc_tuned_shapes() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return (int64_t)g_tuned.size();
}

}  // namespace cq
