// SIMT kernels of the THC-RPA/GW path: fused k<->R DFT + Hadamard products, in-place IR
// transforms, layout conversions, determinants and the dielectric head.
//
// All large arrays are (leading index, ncol) row-major with ncol = Np * Np consecutive
// auxiliary-basis elements, so every kernel reads and writes whole 32-column runs per warp.
#include <atomic>
#include <type_traits>
#include <mutex>

#include "kernels.cuh"

namespace cq {

static std::atomic<int64_t> g_launches{0};
int64_t launches_total() { return g_launches.load(); }
void count_launch(int64_t n) { g_launches += n; }

#define CQ_LAUNCHED() \
  do {                \
    count_launch();   \
    CQ_CHECK_CUDA(cudaGetLastError()); \
  } while (0)

// ---------------------------------------------------------------------------------------
// small DFTs
// ---------------------------------------------------------------------------------------
constexpr int kMaxDftN = 8;
// c_tw[n][r] = exp(-2 pi i r / n)
__constant__ double2 c_tw[kMaxDftN + 1][kMaxDftN];

void upload_twiddles() {
  static std::mutex mu;
  static int done_mask = 0;  // one bit per device ordinal (< 32)
  int dev = 0;
  CQ_CHECK_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 32 && (done_mask >> dev) & 1) return;
  double2 h[kMaxDftN + 1][kMaxDftN] = {};
  const double pi = 3.14159265358979323846;
  for (int n = 1; n <= kMaxDftN; ++n)
    for (int r = 0; r < n; ++r) {
      h[n][r].x = std::cos(2.0 * pi * r / n);
      h[n][r].y = -std::sin(2.0 * pi * r / n);
    }
  // exact values for the quarter turns
  for (int n = 1; n <= kMaxDftN; ++n)
    for (int r = 0; r < n; ++r) {
      if ((4 * r) % n == 0) {
        int q = (4 * r) / n;  // r/n = q/4
        const double cs[4] = {1, 0, -1, 0}, sn[4] = {0, -1, 0, 1};
        h[n][r].x = cs[q & 3];
        h[n][r].y = sn[q & 3];
      }
    }
  CQ_CHECK_CUDA(cudaMemcpyToSymbol(c_tw, h, sizeof(h)));
  if (dev < 32) done_mask |= 1 << dev;
}

// sign i a (sign = +1 or -1)
template <typename C>
__device__ __forceinline__ C mul_si(C a, int sign) {
  C r;
  if (sign > 0) {
    r.x = -a.y;
    r.y = a.x;
  } else {
    r.x = a.y;
    r.y = -a.x;
  }
  return r;
}

// 3-point DFT in place (Winograd's form: 12 real additions, 4 real multiplications):
// y0 = x0 + (x1 + x2), y1,2 = x0 - (x1 + x2)/2 +- sign i (sqrt(3)/2) (x1 - x2)
template <typename C>
__device__ __forceinline__ void dft3pt(C& x0, C& x1, C& x2, int sign) {
  using R = decltype(x0.x);
  const R h = R(0.5), s3 = R(0.86602540378443864676);
  const C t1 = cadd(x1, x2), d = csub(x1, x2);
  C t2, t3;
  t2.x = x0.x - h * t1.x;
  t2.y = x0.y - h * t1.y;
  t3.x = s3 * d.x;
  t3.y = s3 * d.y;
  const C u = mul_si(t3, sign);
  x0 = cadd(x0, t1);
  x1 = cadd(t2, u);
  x2 = csub(t2, u);
}

// y_j = sum_m x_m exp(sign 2 pi i j m / N), in place.  N = 2, 3, 4, 6, 8 in closed form
// (N = 6 as Good-Thomas 2 x 3: input n = (3 n1 + 2 n2) mod 6, output k = (3 k1 + 4 k2) mod 6,
// no twiddles; N = 8 as radix 2 over two 4-point transforms); N = 5, 7 as the plain sum.
template <typename C, int N>
__device__ __forceinline__ void dft_line(C (&x)[N], int sign) {
  if constexpr (N == 1) {
    return;
  } else if constexpr (N == 2) {
    C a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if constexpr (N == 3) {
    dft3pt(x[0], x[1], x[2], sign);
  } else if constexpr (N == 4) {
    C a0 = cadd(x[0], x[2]), a1 = csub(x[0], x[2]);
    C b0 = cadd(x[1], x[3]), b1 = csub(x[1], x[3]);
    const C b1w = mul_si(b1, sign);  // b1 * exp(sign i pi / 2)
    x[0] = cadd(a0, b0);
    x[2] = csub(a0, b0);
    x[1] = cadd(a1, b1w);
    x[3] = csub(a1, b1w);
  } else if constexpr (N == 6) {
    C a0 = x[0], a1 = x[2], a2 = x[4];  // n1 = 0: n = 0, 2, 4
    C b0 = x[3], b1 = x[5], b2 = x[1];  // n1 = 1: n = 3, 5, 1
    dft3pt(a0, a1, a2, sign);
    dft3pt(b0, b1, b2, sign);
    x[0] = cadd(a0, b0);  // (k1, k2) = (0, 0)
    x[3] = csub(a0, b0);  // (1, 0)
    x[4] = cadd(a1, b1);  // (0, 1)
    x[1] = csub(a1, b1);  // (1, 1)
    x[2] = cadd(a2, b2);  // (0, 2)
    x[5] = csub(a2, b2);  // (1, 2)
  } else if constexpr (N == 8) {
    using R = decltype(x[0].x);
    const R h = R(0.70710678118654752440);
    C e[4] = {x[0], x[2], x[4], x[6]}, o[4] = {x[1], x[3], x[5], x[7]};
    dft_line<C, 4>(e, sign);
    dft_line<C, 4>(o, sign);
    // o[k] exp(sign 2 pi i k / 8): k = 1: (1 + sign i)/sqrt2, 2: sign i, 3: (-1 + sign i)/sqrt2
    const R sg = sign > 0 ? R(1) : R(-1);
    C w[4];
    w[0] = o[0];
    w[1].x = h * (o[1].x - sg * o[1].y);
    w[1].y = h * (o[1].y + sg * o[1].x);
    w[2] = mul_si(o[2], sign);
    w[3].x = h * (-o[3].x - sg * o[3].y);
    w[3].y = h * (-o[3].y + sg * o[3].x);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      x[k] = cadd(e[k], w[k]);
      x[k + 4] = csub(e[k], w[k]);
    }
  } else {
    C y[N];
#pragma unroll
    for (int j = 0; j < N; ++j) {
      C acc = x[0];
#pragma unroll
      for (int m = 1; m < N; ++m) {
        const double2 t = c_tw[N][(j * m) % N];
        C w;
        w.x = t.x;
        w.y = sign > 0 ? -t.y : t.y;
        acc = cadd(acc, cmul(x[m], w));
      }
      y[j] = acc;
    }
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = y[j];
  }
}

// One dimension (length N, stride `stride` in k units) of the DFT of a smem tile A[k][TILE].
template <typename C, int TILE, int N>
__device__ __forceinline__ void dft_dim_n(C* A, int stride, int nk, int sign) {
  const int lines = nk / N;
  const int items = lines * TILE;
  for (int i = threadIdx.x; i < items; i += blockDim.x) {
    const int c = i % TILE;
    const int line = i / TILE;
    const int inner = line % stride, outer = line / stride;
    const int k0 = outer * N * stride + inner;
    C x[N];
#pragma unroll
    for (int m = 0; m < N; ++m) x[m] = A[(k0 + m * stride) * TILE + c];
    dft_line<C, N>(x, sign);
#pragma unroll
    for (int m = 0; m < N; ++m) A[(k0 + m * stride) * TILE + c] = x[m];
  }
}

template <typename C, int TILE>
__device__ void dft_dim(C* A, int n, int stride, int nk, int sign) {
  switch (n) {
    case 1: break;
    case 2: dft_dim_n<C, TILE, 2>(A, stride, nk, sign); break;
    case 3: dft_dim_n<C, TILE, 3>(A, stride, nk, sign); break;
    case 4: dft_dim_n<C, TILE, 4>(A, stride, nk, sign); break;
    case 5: dft_dim_n<C, TILE, 5>(A, stride, nk, sign); break;
    case 6: dft_dim_n<C, TILE, 6>(A, stride, nk, sign); break;
    case 7: dft_dim_n<C, TILE, 7>(A, stride, nk, sign); break;
    case 8: dft_dim_n<C, TILE, 8>(A, stride, nk, sign); break;
    default: break;  // rejected on the host
  }
}

// 3D DFT of up to three tiles at once (fewer barriers).
template <typename C, int TILE>
__device__ void dft3(C* A, C* B, int n0, int n1, int n2, int sign) {
  const int nk = n0 * n1 * n2;
  dft_dim<C, TILE>(A, n2, 1, nk, sign);
  if (B) dft_dim<C, TILE>(B, n2, 1, nk, sign);
  __syncthreads();
  dft_dim<C, TILE>(A, n1, n2, nk, sign);
  if (B) dft_dim<C, TILE>(B, n1, n2, nk, sign);
  __syncthreads();
  dft_dim<C, TILE>(A, n0, n1 * n2, nk, sign);
  if (B) dft_dim<C, TILE>(B, n0, n1 * n2, nk, sign);
  __syncthreads();
}

// 3D DFT of one or two tiles on an NC x NC x NC grid known at compile time (NC > 0), else
// the runtime-shaped dft3; constant strides remove the index arithmetic from the loops.
template <typename C, int TILE, int NC>
__device__ __forceinline__ void dft3c(C* A, C* B, int n0, int n1, int n2, int sign) {
  if constexpr (NC == 0) {
    dft3<C, TILE>(A, B, n0, n1, n2, sign);
  } else {
    constexpr int NK = NC * NC * NC;
    if constexpr (NC > 1) {
      dft_dim_n<C, TILE, NC>(A, 1, NK, sign);
      if (B) dft_dim_n<C, TILE, NC>(B, 1, NK, sign);
      __syncthreads();
      dft_dim_n<C, TILE, NC>(A, NC, NK, sign);
      if (B) dft_dim_n<C, TILE, NC>(B, NC, NK, sign);
      __syncthreads();
      dft_dim_n<C, TILE, NC>(A, NC * NC, NK, sign);
      if (B) dft_dim_n<C, TILE, NC>(B, NC * NC, NK, sign);
    }
    __syncthreads();
  }
}

// Tile loads are issued 8 per thread before the shared-memory stores so that enough
// requests are in flight to cover DRAM latency.
template <typename C, int TILE>
__device__ __forceinline__ void load_tile(C* A, const C* __restrict__ src, int nk, int64_t ncol,
                                          int64_t col0) {
  const int total = nk * TILE;
  for (int i0 = 0; i0 < total; i0 += 8 * 256) {
    C v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + threadIdx.x + u * 256;
      const int k = i / TILE, c = i % TILE;
      const int64_t col = col0 + c;
      v[u].x = 0;
      v[u].y = 0;
      if (i < total && col < ncol) v[u] = src[(int64_t)k * ncol + col];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + threadIdx.x + u * 256;
      if (i < total) A[i] = v[u];
    }
  }
}

template <typename C, int TILE>
__device__ __forceinline__ void store_tile(const C* A, C* dst, int nk, int64_t ncol,
                                           int64_t col0) {
  for (int i = threadIdx.x; i < nk * TILE; i += blockDim.x) {
    const int k = i / TILE, c = i % TILE;
    const int64_t col = col0 + c;
    if (col < ncol) dst[(int64_t)k * ncol + col] = A[i];
  }
}

// Compile-time line length for a runtime DFT dimension n (1..8).
template <typename F> __device__ __forceinline__ void with_n(int n, F&& f) {
  switch (n) {
    case 1: f(std::integral_constant<int, 1>{}); break;
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 3: f(std::integral_constant<int, 3>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 5: f(std::integral_constant<int, 5>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 7: f(std::integral_constant<int, 7>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    default: break;  // rejected on the host
  }
}

// One in-shared-memory DFT dimension (the middle one, stride n2) of a tile.
template <typename C, int TILE, int NC>
__device__ __forceinline__ void mid_pass(C* A, int n1, int n2, int nk, int sign) {
  if constexpr (NC > 0) {
    if constexpr (NC > 1) dft_dim_n<C, TILE, NC>(A, NC, NC * NC * NC, sign);
  } else {
    dft_dim<C, TILE>(A, n1, n2, nk, sign);
  }
}

// Global rows (k, ncol apart) -> DFT along the innermost dimension (length N, stride 1 in k)
// in registers -> shared tile A[k][TILE]: the load and the first DFT pass in one sweep.
template <typename C, int TILE, int N>
__device__ __forceinline__ void load_dft_inner(C* A, const C* __restrict__ src, int nk,
                                               int64_t ncol, int64_t col0, int sign) {
  const int lines = nk / N;
  for (int i = threadIdx.x; i < lines * TILE; i += blockDim.x) {
    const int c = i % TILE, line = i / TILE;
    const int64_t col = col0 + c;
    C x[N];
#pragma unroll
    for (int m = 0; m < N; ++m) {
      x[m].x = 0;
      x[m].y = 0;
      if (col < ncol) x[m] = src[(int64_t)(line * N + m) * ncol + col];
    }
    dft_line<C, N>(x, sign);
#pragma unroll
    for (int m = 0; m < N; ++m) A[(line * N + m) * TILE + c] = x[m];
  }
}

// load_dft_inner for two tiles at once (A from srcA, B from srcB, or A alone when srcB is
// null): each thread issues the loads of both lines before either DFT, so twice as many
// loads are in flight while the tiles cross HBM.  Same arithmetic as two load_dft_inner calls.
template <typename C, int TILE, int N>
__device__ __forceinline__ void load_dft_inner2(C* A, const C* __restrict__ srcA, C* B,
                                                const C* __restrict__ srcB, int nk,
                                                int64_t ncol, int64_t col0, int sign) {
  const int lines = nk / N;
  for (int i = threadIdx.x; i < lines * TILE; i += blockDim.x) {
    const int c = i % TILE, line = i / TILE;
    const int64_t col = col0 + c;
    C x[N], y[N];
#pragma unroll
    for (int m = 0; m < N; ++m) {
      x[m].x = 0;
      x[m].y = 0;
      y[m] = x[m];
      if (col < ncol) {
        x[m] = srcA[(int64_t)(line * N + m) * ncol + col];
        if (srcB) y[m] = srcB[(int64_t)(line * N + m) * ncol + col];
      }
    }
    dft_line<C, N>(x, sign);
#pragma unroll
    for (int m = 0; m < N; ++m) A[(line * N + m) * TILE + c] = x[m];
    if (srcB) {
      dft_line<C, N>(y, sign);
#pragma unroll
      for (int m = 0; m < N; ++m) B[(line * N + m) * TILE + c] = y[m];
    }
  }
}

// Shared tile -> DFT along the innermost dimension in registers -> global rows: the last DFT
// pass and the store in one sweep.
template <typename C, int TILE, int N>
__device__ __forceinline__ void dft_inner_store(const C* A, C* dst, int nk, int64_t ncol,
                                                int64_t col0, int sign) {
  const int lines = nk / N;
  for (int i = threadIdx.x; i < lines * TILE; i += blockDim.x) {
    const int c = i % TILE, line = i / TILE;
    const int64_t col = col0 + c;
    C x[N];
#pragma unroll
    for (int m = 0; m < N; ++m) x[m] = A[(line * N + m) * TILE + c];
    dft_line<C, N>(x, sign);
    if (col < ncol) {
#pragma unroll
      for (int m = 0; m < N; ++m) dst[(int64_t)(line * N + m) * ncol + col] = x[m];
    }
  }
}

// The outermost dimension (length N, stride `stride` = n1 n2): pre(w, k_inner, c) issues the
// global loads of the line's third operand first, then the forward DFT of the A (and B) lines,
// op(a, b, w) on them in registers, inverse DFT of A (and, if inv_b, B), back to shared memory:
// the last forward pass, the pointwise product and the first inverse pass in one sweep.
template <typename C, int TILE, int N, typename Pre, typename Op>
__device__ __forceinline__ void outer_pointwise(C* A, C* B, bool inv_b, int stride, Pre&& pre,
                                                Op&& op) {
  for (int i = threadIdx.x; i < stride * TILE; i += blockDim.x) {
    const int c = i % TILE, inner = i / TILE;
    C a[N], b[N], w[N];
    pre(w, inner, c);  // global loads of the line's operand, in flight during the DFT below
#pragma unroll
    for (int m = 0; m < N; ++m) a[m] = A[(inner + m * stride) * TILE + c];
    if (B) {
#pragma unroll
      for (int m = 0; m < N; ++m) b[m] = B[(inner + m * stride) * TILE + c];
      dft_line<C, N>(b, -1);
    }
    dft_line<C, N>(a, -1);
    op(a, b, w);
    dft_line<C, N>(a, +1);
#pragma unroll
    for (int m = 0; m < N; ++m) A[(inner + m * stride) * TILE + c] = a[m];
    if (B && inv_b) {
      dft_line<C, N>(b, +1);
#pragma unroll
      for (int m = 0; m < N; ++m) B[(inner + m * stride) * TILE + c] = b[m];
    }
  }
}

// The (n1, n2) plane of one column at outer index i0 of an N x N x N grid, held in registers:
// DFT along the innermost dimension (N lines of N consecutive k), then along the middle one
// (lines of stride N).  Forward: global rows -> plane -> shared tile A[k][TILE]; inverse:
// shared tile -> plane (middle, then innermost) -> global rows.  The same dft_line calls in
// the same order as the load + middle sweeps of the shared-memory form, without the two
// shared-memory sweeps of the middle dimension.
template <typename C, int N, bool MIDDLE_FIRST>
__device__ __forceinline__ void plane_dft(C (&x)[N * N], int sign) {
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
    const bool inner = (pass == 0) != MIDDLE_FIRST;
#pragma unroll
    for (int l = 0; l < N; ++l) {
      C y[N];
#pragma unroll
      for (int m = 0; m < N; ++m) y[m] = x[inner ? l * N + m : l + m * N];
      dft_line<C, N>(y, sign);
#pragma unroll
      for (int m = 0; m < N; ++m) x[inner ? l * N + m : l + m * N] = y[m];
    }
  }
}

template <typename C, int TILE, int N>
__device__ __forceinline__ void plane_load_dft(C* A, const C* __restrict__ src, int i0, int c,
                                               int64_t ncol, int64_t col0, int sign) {
  constexpr int P = N * N;
  const int64_t col = col0 + c;
  C x[P];
  const C* p = src + (int64_t)i0 * P * ncol + col;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    x[j].x = 0;
    x[j].y = 0;
    if (col < ncol) x[j] = p[0];
    p += ncol;
  }
  plane_dft<C, N, false>(x, sign);
#pragma unroll
  for (int j = 0; j < P; ++j) A[(i0 * P + j) * TILE + c] = x[j];
}

template <typename C, int TILE, int N>
__device__ __forceinline__ void plane_dft_store(const C* A, C* dst, int i0, int c, int64_t ncol,
                                                int64_t col0, int sign) {
  constexpr int P = N * N;
  const int64_t col = col0 + c;
  C x[P];
#pragma unroll
  for (int j = 0; j < P; ++j) x[j] = A[(i0 * P + j) * TILE + c];
  plane_dft<C, N, true>(x, sign);
  if (col < ncol) {
    C* p = dst + (int64_t)i0 * P * ncol + col;
#pragma unroll
    for (int j = 0; j < P; ++j) {
      p[0] = x[j];
      p += ncol;
    }
  }
}

// k_pi_fused on an N x N x N grid with the middle dimension in registers: 2 N TILE threads,
// thread (h, i0, c) owns the plane (i0, c) of tile h (A = Gp, B = Gn).  Two shared-memory
// sweeps per tile: the outermost DFT + product + inverse, and the inverse planes.
template <typename R, int TILE, int NC>
__global__ void __launch_bounds__(2 * NC * TILE) k_pi_plane(const cplx_t<R>* __restrict__ Gp,
                                                           const cplx_t<R>* __restrict__ Gn,
                                                           cplx_t<R>* __restrict__ Pi,
                                                           int64_t ncol, R scale) {
  using C = cplx_t<R>;
  constexpr int P = NC * NC, NK = NC * P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* A = reinterpret_cast<C*>(smem_raw);
  C* B = A + NK * TILE;
  const int h = threadIdx.x / (NC * TILE), r = threadIdx.x % (NC * TILE);
  const int i0 = r / TILE, c = r % TILE;
  const int64_t ntiles = (ncol + TILE - 1) / TILE;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t col0 = t * TILE;
    plane_load_dft<C, TILE, NC>(h ? B : A, h ? Gn : Gp, i0, c, ncol, col0, -1);
    __syncthreads();
    outer_pointwise<C, TILE, NC>(A, B, false, P, [](C (&)[NC], int, int) {},
                                 [&](C (&a)[NC], C (&b)[NC], C (&)[NC]) {
#pragma unroll
      for (int m = 0; m < NC; ++m) a[m] = cscale(cmulc(a[m], b[m]), scale);
    });
    __syncthreads();
    if (h == 0) plane_dft_store<C, TILE, NC>(A, Pi, i0, c, ncol, col0, +1);
    __syncthreads();
  }
}

// 8-byte asynchronous global -> shared copy; src_bytes = 0 writes zeros and reads nothing.
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Asynchronous copy of the W tile W[k][col0 .. col0 + TILE) into Wt[k][TILE] (zeros past ncol).
template <typename C, int TILE, int NK>
__device__ __forceinline__ void w_tile_async(C* Wt, const C* WR, int64_t ncol, int64_t col0) {
  for (int i = threadIdx.x; i < NK * TILE; i += blockDim.x) {
    const int k = i / TILE, cc = i % TILE;
    const int64_t col = col0 + cc;
    const bool in = col < ncol;
    cp_async8(Wt + i, in ? WR + (int64_t)k * ncol + col : WR, in ? 8 : 0);
  }
  cp_async_commit();
}

// k_sigma_fused on an N x N x N grid with the middle dimension in registers (threads as in
// k_pi_plane; the B half idles when Gm is null).  The W tile of the next column tile streams
// into shared memory (cp.async) while this tile's planes are transformed and stored, so every
// global load of a tile is in flight in one phase.  In place (S may alias G).
template <typename R, int TILE, int NC>
__global__ void __launch_bounds__(2 * NC * TILE) k_sigma_plane(const cplx_t<R>* Gp,
                                                              const cplx_t<R>* Gm,
                                                              const cplx_t<R>* __restrict__ WR,
                                                              cplx_t<R>* Sp, cplx_t<R>* Sm,
                                                              int64_t ncol, R scale) {
  using C = cplx_t<R>;
  constexpr int P = NC * NC, NK = NC * P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* A = reinterpret_cast<C*>(smem_raw);
  C* B = A + NK * TILE;
  C* Wt = B + NK * TILE;
  const bool has_m = (Gm != nullptr);
  const int h = threadIdx.x / (NC * TILE), r = threadIdx.x % (NC * TILE);
  const int i0 = r / TILE, c = r % TILE;
  const bool owns = (h == 0) || has_m;
  const int64_t ntiles = (ncol + TILE - 1) / TILE;
  if (blockIdx.x < ntiles) w_tile_async<C, TILE, NK>(Wt, WR, ncol, (int64_t)blockIdx.x * TILE);
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t col0 = t * TILE;
    if (owns) plane_load_dft<C, TILE, NC>(h ? B : A, h ? Gm : Gp, i0, c, ncol, col0, -1);
    cp_async_wait_all();
    __syncthreads();
    outer_pointwise<C, TILE, NC>(A, has_m ? B : nullptr, true, P,
                                 [&](C (&w)[NC], int inner, int cc) {
#pragma unroll
      for (int m = 0; m < NC; ++m) w[m] = Wt[(inner + m * P) * TILE + cc];
    }, [&](C (&a)[NC], C (&b)[NC], C (&w)[NC]) {
#pragma unroll
      for (int m = 0; m < NC; ++m) {
        const C ws = cscale(w[m], scale);
        a[m] = cmul(a[m], ws);
        if (has_m) b[m] = cmul(b[m], ws);
      }
    });
    __syncthreads();
    const int64_t tn = t + gridDim.x;
    if (tn < ntiles) w_tile_async<C, TILE, NK>(Wt, WR, ncol, tn * TILE);
    if (owns) plane_dft_store<C, TILE, NC>(h ? B : A, h ? Sm : Sp, i0, c, ncol, col0, +1);
    __syncthreads();
  }
}

// k_dft_plain on an N x N x N grid: N TILE threads, one register plane each, then the
// outermost dimension from shared memory straight to the global rows (scaled).
template <typename R, int TILE, int NC>
__global__ void __launch_bounds__(NC * TILE) k_dft_plane(cplx_t<R>* __restrict__ buf,
                                                        int64_t ncol, int sign, R scale,
                                                        int64_t nbatch, int64_t bstride) {
  using C = cplx_t<R>;
  constexpr int P = NC * NC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* A = reinterpret_cast<C*>(smem_raw);
  const int i0 = threadIdx.x / TILE, c = threadIdx.x % TILE;
  const int64_t ntiles = (ncol + TILE - 1) / TILE;
  for (int64_t t = blockIdx.x; t < ntiles * nbatch; t += gridDim.x) {
    const int64_t b = t / ntiles;
    const int64_t col0 = (t % ntiles) * TILE;
    C* base = buf + b * bstride;
    plane_load_dft<C, TILE, NC>(A, base, i0, c, ncol, col0, sign);
    __syncthreads();
    for (int i = threadIdx.x; i < P * TILE; i += blockDim.x) {
      const int cc = i % TILE, inner = i / TILE;
      const int64_t col = col0 + cc;
      C x[NC];
#pragma unroll
      for (int m = 0; m < NC; ++m) x[m] = A[(inner + m * P) * TILE + cc];
      dft_line<C, NC>(x, sign);
      if (col < ncol) {
#pragma unroll
        for (int m = 0; m < NC; ++m) base[(int64_t)(inner + m * P) * ncol + col] = cscale(x[m], scale);
      }
    }
    __syncthreads();
  }
}

// Pi(t) columns: Pi = f_qR[ scale Gp(R) o conj(Gn(R)) ] with G(R) = f_Rk G(k), four shared-
// memory sweeps per tile (load + innermost DFT, middle DFT, outermost DFT + product + inverse,
// middle inverse, innermost inverse + store).
template <typename R, int TILE, int NC>
__global__ void __launch_bounds__(256) k_pi_fused(const cplx_t<R>* __restrict__ Gp,
                                                  const cplx_t<R>* __restrict__ Gn,
                                                  cplx_t<R>* __restrict__ Pi, int64_t ncol,
                                                  int rn0, int rn1, int rn2, R scale) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n0 = NC ? NC : rn0, n1 = NC ? NC : rn1, n2 = NC ? NC : rn2;
  const int nk = n0 * n1 * n2;
  C* A = reinterpret_cast<C*>(smem_raw);
  C* B = A + nk * TILE;
  const int64_t ntiles = (ncol + TILE - 1) / TILE;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t col0 = t * TILE;
    with_n(n2, [&](auto N2) {
      load_dft_inner2<C, TILE, decltype(N2)::value>(A, Gp, B, Gn, nk, ncol, col0, -1);
    });
    __syncthreads();
    mid_pass<C, TILE, NC>(A, n1, n2, nk, -1);
    mid_pass<C, TILE, NC>(B, n1, n2, nk, -1);
    __syncthreads();
    with_n(n0, [&](auto N0) {
      constexpr int N = decltype(N0)::value;
      outer_pointwise<C, TILE, N>(A, B, false, n1 * n2, [](C (&)[N], int, int) {},
                                  [&](C (&a)[N], C (&b)[N], C (&)[N]) {
#pragma unroll
        for (int m = 0; m < N; ++m) a[m] = cscale(cmulc(a[m], b[m]), scale);
      });
    });
    __syncthreads();
    mid_pass<C, TILE, NC>(A, n1, n2, nk, +1);
    __syncthreads();
    with_n(n2, [&](auto N2) {
      dft_inner_store<C, TILE, decltype(N2)::value>(A, Pi, nk, ncol, col0, +1);
    });
    __syncthreads();
  }
}

// Sigma(t) columns (both halves): S = f_kR[ -(f_Rk G) o W_R ] (scale = -1/nk), W_R read from
// global memory inside the outermost-dimension sweep.  In place (S may alias G).
template <typename R, int TILE, int NC>
__global__ void __launch_bounds__(256) k_sigma_fused(const cplx_t<R>* Gp, const cplx_t<R>* Gm,
                                                     const cplx_t<R>* __restrict__ WR,
                                                     cplx_t<R>* Sp, cplx_t<R>* Sm, int64_t ncol,
                                                     int rn0, int rn1, int rn2, R scale) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n0 = NC ? NC : rn0, n1 = NC ? NC : rn1, n2 = NC ? NC : rn2;
  const int nk = n0 * n1 * n2;
  C* A = reinterpret_cast<C*>(smem_raw);
  C* B = A + nk * TILE;
  const bool has_m = (Gm != nullptr);
  const int64_t ntiles = (ncol + TILE - 1) / TILE;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t col0 = t * TILE;
    with_n(n2, [&](auto N2) {
      load_dft_inner2<C, TILE, decltype(N2)::value>(A, Gp, B, has_m ? Gm : nullptr, nk, ncol,
                                                    col0, -1);
    });
    __syncthreads();
    mid_pass<C, TILE, NC>(A, n1, n2, nk, -1);
    if (has_m) mid_pass<C, TILE, NC>(B, n1, n2, nk, -1);
    __syncthreads();
    const int stride = n1 * n2;
    with_n(n0, [&](auto N0) {
      constexpr int N = decltype(N0)::value;
      outer_pointwise<C, TILE, N>(A, has_m ? B : nullptr, true, stride,
                                  [&](C (&w)[N], int inner, int c) {
        const int64_t col = col0 + c;
#pragma unroll
        for (int m = 0; m < N; ++m) {
          w[m].x = 0;
          w[m].y = 0;
          if (col < ncol) w[m] = WR[(int64_t)(inner + m * stride) * ncol + col];
        }
      }, [&](C (&a)[N], C (&b)[N], C (&w)[N]) {
#pragma unroll
        for (int m = 0; m < N; ++m) {
          const C ws = cscale(w[m], scale);
          a[m] = cmul(a[m], ws);
          if (has_m) b[m] = cmul(b[m], ws);
        }
      });
    });
    __syncthreads();
    mid_pass<C, TILE, NC>(A, n1, n2, nk, +1);
    if (has_m) mid_pass<C, TILE, NC>(B, n1, n2, nk, +1);
    __syncthreads();
    with_n(n2, [&](auto N2) {
      dft_inner_store<C, TILE, decltype(N2)::value>(A, Sp, nk, ncol, col0, +1);
      if (has_m) dft_inner_store<C, TILE, decltype(N2)::value>(B, Sm, nk, ncol, col0, +1);
    });
    __syncthreads();
  }
}

template <typename R, int TILE, int NC>
__global__ void __launch_bounds__(256) k_dft_plain(cplx_t<R>* __restrict__ buf, int64_t ncol,
                                                   int rn0, int rn1, int rn2, int sign, R scale,
                                                   int64_t nbatch, int64_t bstride) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n0 = NC ? NC : rn0, n1 = NC ? NC : rn1, n2 = NC ? NC : rn2;
  const int nk = n0 * n1 * n2;
  C* A = reinterpret_cast<C*>(smem_raw);
  const int64_t ntiles = (ncol + TILE - 1) / TILE;
  for (int64_t t = blockIdx.x; t < ntiles * nbatch; t += gridDim.x) {
    const int64_t b = t / ntiles;
    const int64_t col0 = (t % ntiles) * TILE;
    C* base = buf + b * bstride;
    load_tile<C, TILE>(A, base, nk, ncol, col0);
    __syncthreads();
    dft3c<C, TILE, NC>(A, (C*)nullptr, n0, n1, n2, sign);
    for (int i = threadIdx.x; i < nk * TILE; i += blockDim.x) A[i] = cscale(A[i], scale);
    __syncthreads();
    store_tile<C, TILE>(A, base, nk, ncol, col0);
    __syncthreads();
  }
}

template <typename R>
static int pick_tile(int nk) {
  // keep at most ~96 KB of tiles per block (three tiles in the sigma kernel)
  const int64_t per32 = (int64_t)nk * 32 * sizeof(cplx_t<R>) * 3;
  return per32 <= 96 * 1024 ? 32 : 16;
}

// Register-plane forms of the column kernels: complex64 on cubic grids with edge > 1 (a plane
// of edge^2 complex64 values per thread); complex128 and other grids keep the shared-memory form.
template <typename R, int NC> constexpr bool use_plane() { return sizeof(R) == 4 && NC > 1; }

static void check_grid(KGrid g) {
  CQ_REQUIRE(g.n0 >= 1 && g.n1 >= 1 && g.n2 >= 1 && g.n0 <= kMaxDftN && g.n1 <= kMaxDftN &&
                 g.n2 <= kMaxDftN,
             COQUI_B200_EUNSUPPORTED, "k-grid edges must be in [1, 8]");
}

static void set_smem(const void* fn, size_t bytes) {
  if (bytes > 48 * 1024)
    CQ_CHECK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// cubic grid edge compiled as a constant (0 = runtime shape)
static int cubic_edge(KGrid g) {
  if (g.n0 == g.n1 && g.n1 == g.n2 && (g.n0 == 1 || g.n0 == 2 || g.n0 == 3 || g.n0 == 4 || g.n0 == 6))
    return g.n0;
  return 0;
}

#define CQ_DISPATCH_NC(g, ...)                 \
  switch (cubic_edge(g)) {                     \
    case 1: { constexpr int NCV = 1; __VA_ARGS__; } break; \
    case 2: { constexpr int NCV = 2; __VA_ARGS__; } break; \
    case 3: { constexpr int NCV = 3; __VA_ARGS__; } break; \
    case 4: { constexpr int NCV = 4; __VA_ARGS__; } break; \
    case 6: { constexpr int NCV = 6; __VA_ARGS__; } break; \
    default: { constexpr int NCV = 0; __VA_ARGS__; } break; \
  }

// One k-point (Gamma-only): every DFT is the identity and the column kernels reduce to
// element-wise products; these stream the arrays at full width instead of staging 32-column
// tiles through shared memory.
template <typename R>
__global__ void __launch_bounds__(256) k_pi_gamma(const cplx_t<R>* __restrict__ Gp,
                                                  const cplx_t<R>* __restrict__ Gn,
                                                  cplx_t<R>* __restrict__ Pi, int64_t n, R scale) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    Pi[i] = cscale(cmulc(Gp[i], Gn[i]), scale);
}
template <typename R>
__global__ void __launch_bounds__(256) k_sigma_gamma(const cplx_t<R>* Gp, const cplx_t<R>* Gm,
                                                     const cplx_t<R>* __restrict__ WR,
                                                     cplx_t<R>* Sp, cplx_t<R>* Sm, int64_t n,
                                                     R scale) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const cplx_t<R> w = cscale(WR[i], scale);
    Sp[i] = cmul(Gp[i], w);
    if (Gm) Sm[i] = cmul(Gm[i], w);
  }
}
template <typename R>
__global__ void __launch_bounds__(256) k_scale_batch(cplx_t<R>* buf, int64_t ncol, int64_t nbatch,
                                                     int64_t bstride, R scale) {
  const int64_t n = ncol * nbatch;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    cplx_t<R>* p = buf + (i / ncol) * bstride + i % ncol;
    *p = cscale(*p, scale);
  }
}

template <typename R>
void launch_pi_fused(const cplx_t<R>* Gp, const cplx_t<R>* Gn, cplx_t<R>* Pi, int64_t ncol,
                     KGrid g, double sp, cudaStream_t s) {
  check_grid(g);
  const int nk = g.nk();
  const R scale = (R)(sp / ((double)nk * (double)nk));
  if (nk == 1) {
    k_pi_gamma<R><<<grid_for(ncol, 256), 256, 0, s>>>(Gp, Gn, Pi, ncol, scale);
    CQ_LAUNCHED();
    return;
  }
  const int tile = pick_tile<R>(nk);
  const size_t smem = (size_t)2 * nk * tile * sizeof(cplx_t<R>);
  const int64_t ntiles = (ncol + tile - 1) / tile;
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, 148 * 16);
#define CQ_PI_LAUNCH(T)                                                                    \
  CQ_DISPATCH_NC(g, if constexpr (use_plane<R, NCV>()) {                                     \
    set_smem((const void*)k_pi_plane<R, T, NCV>, smem);                                      \
    k_pi_plane<R, T, NCV><<<grid, 2 * NCV * T, smem, s>>>(Gp, Gn, Pi, ncol, scale);          \
  } else {                                                                                   \
    set_smem((const void*)k_pi_fused<R, T, NCV>, smem);                                      \
    k_pi_fused<R, T, NCV><<<grid, 256, smem, s>>>(Gp, Gn, Pi, ncol, g.n0, g.n1, g.n2, scale); \
  })
  if (tile == 32) {
    CQ_PI_LAUNCH(32)
  } else {
    CQ_PI_LAUNCH(16)
  }
#undef CQ_PI_LAUNCH
  CQ_LAUNCHED();
}

template <typename R>
void launch_sigma_fused(const cplx_t<R>* Gp, const cplx_t<R>* Gm, const cplx_t<R>* WR,
                        cplx_t<R>* Sp, cplx_t<R>* Sm, int64_t ncol, KGrid g, cudaStream_t s) {
  check_grid(g);
  const int nk = g.nk();
  // Sigma = f_kR [ -(f_Rk G) * W_R ]; f_Rk carries 1/nk
  const R scale = (R)(-1.0 / (double)nk);
  if (nk == 1) {
    k_sigma_gamma<R><<<grid_for(ncol, 256), 256, 0, s>>>(Gp, Gm, WR, Sp, Sm, ncol, scale);
    CQ_LAUNCHED();
    return;
  }
  const int tile = pick_tile<R>(nk);
  const size_t smem = (size_t)2 * nk * tile * sizeof(cplx_t<R>);
  const int64_t ntiles = (ncol + tile - 1) / tile;
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, 148 * 16);
#define CQ_SIGMA_LAUNCH(T)                                                                  \
  CQ_DISPATCH_NC(g, if constexpr (use_plane<R, NCV>()) {                                      \
    const size_t smem3 = smem / 2 * 3; /* G+, G- and W tiles */                               \
    set_smem((const void*)k_sigma_plane<R, T, NCV>, smem3);                                   \
    k_sigma_plane<R, T, NCV><<<grid, 2 * NCV * T, smem3, s>>>(Gp, Gm, WR, Sp, Sm, ncol, scale); \
  } else {                                                                                    \
    set_smem((const void*)k_sigma_fused<R, T, NCV>, smem);                                    \
    k_sigma_fused<R, T, NCV><<<grid, 256, smem, s>>>(Gp, Gm, WR, Sp, Sm, ncol, g.n0, g.n1,    \
                                                     g.n2, scale);                            \
  })
  if (tile == 32) {
    CQ_SIGMA_LAUNCH(32)
  } else {
    CQ_SIGMA_LAUNCH(16)
  }
#undef CQ_SIGMA_LAUNCH
  CQ_LAUNCHED();
}

template <typename R>
void launch_dft_plain(cplx_t<R>* buf, int64_t ncol, KGrid g, int sign, double scale,
                      int64_t nbatch, int64_t bstride, cudaStream_t s) {
  check_grid(g);
  const int nk = g.nk();
  if (nk == 1) {  // a length-1 DFT: only the scale
    if (scale != 1.0) {
      k_scale_batch<R><<<grid_for(ncol * nbatch, 256), 256, 0, s>>>(buf, ncol, nbatch, bstride,
                                                                     (R)scale);
      CQ_LAUNCHED();
    }
    return;
  }
  // The register-plane form streams 32-column tiles (256-byte row segments): at 216 k and
  // N_mu 1024 it moves 5.9 TB/s there against 3.9 TB/s with 16 columns.
  const int edge = cubic_edge(g);
  const bool plane = sizeof(R) == 4 && edge > 1;
  const int tile = plane ? 32 : pick_tile<R>(nk);
  const size_t smem = (size_t)nk * tile * sizeof(cplx_t<R>);
  const int64_t ntiles = (ncol + tile - 1) / tile * nbatch;
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, 148 * 16);
#define CQ_DFT_LAUNCH(T)                                                                   \
  CQ_DISPATCH_NC(g, if constexpr (use_plane<R, NCV>()) {                                     \
    set_smem((const void*)k_dft_plane<R, T, NCV>, smem);                                     \
    k_dft_plane<R, T, NCV><<<grid, NCV * T, smem, s>>>(buf, ncol, sign, (R)scale, nbatch,     \
                                                       bstride);                             \
  } else {                                                                                   \
    set_smem((const void*)k_dft_plain<R, T, NCV>, smem);                                     \
    k_dft_plain<R, T, NCV><<<grid, 256, smem, s>>>(buf, ncol, g.n0, g.n1, g.n2, sign,         \
                                                   (R)scale, nbatch, bstride);               \
  })
  if (tile == 32) {
    CQ_DFT_LAUNCH(32)
  } else {
    CQ_DFT_LAUNCH(16)
  }
#undef CQ_DFT_LAUNCH
  CQ_LAUNCHED();
}

// ---------------------------------------------------------------------------------------
// IR transforms along the leading (tau or iw) index, in place, FP64 accumulation
// ---------------------------------------------------------------------------------------
template <typename R, int MAXT>
__global__ void __launch_bounds__(128) k_ir_transform(cplx_t<R>* __restrict__ buf, int64_t ncol,
                                                      int n_in, int n_out,
                                                      const double2* __restrict__ M) {
  extern __shared__ double2 sM[];
  for (int i = threadIdx.x; i < n_in * n_out; i += blockDim.x) sM[i] = M[i];
  __syncthreads();
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ncol;
       e += (int64_t)gridDim.x * blockDim.x) {
    double2 x[MAXT];
#pragma unroll
    for (int t = 0; t < MAXT; ++t) {
      if (t < n_in) {
        const cplx_t<R> v = buf[(int64_t)t * ncol + e];
        x[t].x = v.x;
        x[t].y = v.y;
      } else {
        x[t].x = 0;
        x[t].y = 0;
      }
    }
    for (int n = 0; n < n_out; n += 2) {
      const bool two = n + 1 < n_out;
      double ar = 0, ai = 0, br = 0, bi = 0, cr = 0, ci = 0, dr = 0, di = 0;
      const double2* row = sM + n * n_in;
      const double2* row2 = sM + (two ? n + 1 : n) * n_in;
#pragma unroll
      for (int t = 0; t < MAXT; ++t) {
        if (t < n_in) {
          const double2 m = row[t], m2 = row2[t];
          ar = fma(m.x, x[t].x, ar);
          br = fma(-m.y, x[t].y, br);
          ai = fma(m.x, x[t].y, ai);
          bi = fma(m.y, x[t].x, bi);
          cr = fma(m2.x, x[t].x, cr);
          dr = fma(-m2.y, x[t].y, dr);
          ci = fma(m2.x, x[t].y, ci);
          di = fma(m2.y, x[t].x, di);
        }
      }
      cplx_t<R> o;
      o.x = (R)(ar + br);
      o.y = (R)(ai + bi);
      buf[(int64_t)n * ncol + e] = o;
      if (two) {
        o.x = (R)(cr + dr);
        o.y = (R)(ci + di);
        buf[(int64_t)(n + 1) * ncol + e] = o;
      }
    }
  }
}

template <typename R>
void launch_ir_transform(cplx_t<R>* buf, int64_t ncol, int n_in, int n_out, const double2* M,
                         cudaStream_t s) {
  CQ_REQUIRE(n_in >= 1 && n_in <= 96 && n_out >= 1, COQUI_B200_EUNSUPPORTED,
             "IR transform supports at most 96 input points");
  const size_t smem = (size_t)n_in * n_out * sizeof(double2);
  const unsigned grid = grid_for(ncol, 128, 148 * 32);
  if (n_in <= 32) {
    set_smem((const void*)k_ir_transform<R, 32>, smem);
    k_ir_transform<R, 32><<<grid, 128, smem, s>>>(buf, ncol, n_in, n_out, M);
  } else {
    set_smem((const void*)k_ir_transform<R, 96>, smem);
    k_ir_transform<R, 96><<<grid, 128, smem, s>>>(buf, ncol, n_in, n_out, M);
  }
  CQ_LAUNCHED();
}

// Real transform matrix (the particle-hole symmetric IR matrices are real): four outputs
// per pass, 2 FP64 FMAs per (output, input) pair.
template <typename R, int MAXT>
__global__ void __launch_bounds__(128) k_ir_transform_real(cplx_t<R>* __restrict__ buf,
                                                           int64_t ncol, int n_in, int n_out,
                                                           const double* __restrict__ M) {
  extern __shared__ double sMr[];
  for (int i = threadIdx.x; i < n_in * n_out; i += blockDim.x) sMr[i] = M[i];
  __syncthreads();
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ncol;
       e += (int64_t)gridDim.x * blockDim.x) {
    double2 x[MAXT];
#pragma unroll
    for (int t = 0; t < MAXT; ++t) {
      if (t < n_in) {
        const cplx_t<R> v = buf[(int64_t)t * ncol + e];
        x[t].x = v.x;
        x[t].y = v.y;
      } else {
        x[t].x = 0;
        x[t].y = 0;
      }
    }
    for (int n = 0; n < n_out; n += 4) {
      double acc[4][2] = {};
      const double* rows[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) rows[q] = sMr + (n + q < n_out ? n + q : n) * n_in;
#pragma unroll
      for (int t = 0; t < MAXT; ++t) {
        if (t < n_in) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const double m = rows[q][t];
            acc[q][0] = fma(m, x[t].x, acc[q][0]);
            acc[q][1] = fma(m, x[t].y, acc[q][1]);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (n + q < n_out) {
          cplx_t<R> o;
          o.x = (R)acc[q][0];
          o.y = (R)acc[q][1];
          buf[(int64_t)(n + q) * ncol + e] = o;
        }
    }
  }
}

// Complex64 storage with FP32 accumulation (mixed-precision form): the 2 n_in FMAs per output
// then cost half the FP64 form's issue slots, so the transform stays bound by its HBM
// traffic.  The accumulation error is of the order of the complex64 rounding of the inputs
// (the IR rows are sums of same-sign weights for the low frequencies, at most |T| ~ 1e3).
// M (n_out, n_in) FP64 is staged into shared memory as FP32, rows padded to MAXT entries and
// the row count to a multiple of 4 with zeros, so that one float4 read feeds 8 FMAs.
template <int MAXT>
__global__ void __launch_bounds__(128) k_ir_transform_f32(float2* __restrict__ buf, int64_t ncol,
                                                          int n_in, int n_out,
                                                          const double* __restrict__ M) {
  static_assert(MAXT % 4 == 0, "MAXT must be a multiple of 4");
  extern __shared__ float4 sM4[];
  float* sMf = reinterpret_cast<float*>(sM4);
  const int n_out4 = (n_out + 3) / 4;
  for (int i = threadIdx.x; i < n_out4 * 4 * MAXT; i += blockDim.x) {
    const int o = i / MAXT, t = i % MAXT;
    sMf[i] = (o < n_out && t < n_in) ? (float)M[o * n_in + t] : 0.f;
  }
  __syncthreads();
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ncol;
       e += (int64_t)gridDim.x * blockDim.x) {
    float2 x[MAXT];
#pragma unroll
    for (int t = 0; t < MAXT; ++t)
      x[t] = (t < n_in) ? buf[(int64_t)t * ncol + e] : make_float2(0.f, 0.f);
    for (int o4 = 0; o4 < n_out4; ++o4) {
      // (re, im) accumulated together by the packed FP32 FMA of sm_100 (one instruction per
      // complex multiply-add by a real coefficient; each half rounds as fmaf does)
      float2 acc[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = make_float2(0.f, 0.f);
      const float4* rows = sM4 + (size_t)o4 * 4 * (MAXT / 4);
#pragma unroll
      for (int t4 = 0; t4 < MAXT / 4; ++t4) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 m = rows[q * (MAXT / 4) + t4];
          acc[q] = __ffma2_rn(make_float2(m.x, m.x), x[4 * t4 + 0], acc[q]);
          acc[q] = __ffma2_rn(make_float2(m.y, m.y), x[4 * t4 + 1], acc[q]);
          acc[q] = __ffma2_rn(make_float2(m.z, m.z), x[4 * t4 + 2], acc[q]);
          acc[q] = __ffma2_rn(make_float2(m.w, m.w), x[4 * t4 + 3], acc[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (o4 * 4 + q < n_out) __stcs(buf + (int64_t)(o4 * 4 + q) * ncol + e, acc[q]);
    }
  }
}

template <int MAXT>
static void launch_ir_f32(float2* buf, int64_t ncol, int n_in, int n_out, const double* M,
                          cudaStream_t s) {
  const size_t smem = (size_t)((n_out + 3) / 4) * 4 * MAXT * sizeof(float);
  // 128-thread blocks: five resident per SM at 96 registers (two of 256 threads) overlap one
  // block's loads with another's arithmetic (5.19 against 4.94 TB/s for 31 -> 31 points)
  set_smem((const void*)k_ir_transform_f32<MAXT>, smem);
  k_ir_transform_f32<MAXT><<<grid_for(ncol, 128, 148 * 32), 128, smem, s>>>(buf, ncol, n_in, n_out, M);
  CQ_LAUNCHED();
}

template <typename R>
void launch_ir_transform_real(cplx_t<R>* buf, int64_t ncol, int n_in, int n_out, const double* M,
                              cudaStream_t s) {
  CQ_REQUIRE(n_in >= 1 && n_in <= 96 && n_out >= 1, COQUI_B200_EUNSUPPORTED,
             "IR transform supports at most 96 input points");
  if constexpr (std::is_same<R, float>::value) {
    float2* b = reinterpret_cast<float2*>(buf);
    if (n_in <= 16) return launch_ir_f32<16>(b, ncol, n_in, n_out, M, s);
    if (n_in <= 24) return launch_ir_f32<24>(b, ncol, n_in, n_out, M, s);
    if (n_in <= 32) return launch_ir_f32<32>(b, ncol, n_in, n_out, M, s);
    if (n_in <= 48) return launch_ir_f32<48>(b, ncol, n_in, n_out, M, s);
  }
  const size_t smem = (size_t)n_in * n_out * sizeof(double);
  const unsigned grid = grid_for(ncol, 128, 148 * 32);
  if (n_in <= 32) {
    set_smem((const void*)k_ir_transform_real<R, 32>, smem);
    k_ir_transform_real<R, 32><<<grid, 128, smem, s>>>(buf, ncol, n_in, n_out, M);
  } else {
    set_smem((const void*)k_ir_transform_real<R, 96>, smem);
    k_ir_transform_real<R, 96><<<grid, 128, smem, s>>>(buf, ncol, n_in, n_out, M);
  }
  CQ_LAUNCHED();
}

// ---------------------------------------------------------------------------------------
// conversions, layout changes
// ---------------------------------------------------------------------------------------
template <typename R>
__global__ void k_from_c128(const double2* __restrict__ in, cplx_t<R>* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = in[i];
    cplx_t<R> o;
    o.x = (R)v.x;
    o.y = (R)v.y;
    out[i] = o;
  }
}
template <typename R>
__global__ void k_to_c128(const cplx_t<R>* __restrict__ in, double2* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const cplx_t<R> v = in[i];
    out[i] = make_double2(v.x, v.y);
  }
}
template <typename R>
void launch_from_c128(const double2* in, cplx_t<R>* out, int64_t n, cudaStream_t s) {
  k_from_c128<R><<<grid_for(n, 256), 256, 0, s>>>(in, out, n);
  CQ_LAUNCHED();
}
template <typename R>
void launch_to_c128(const cplx_t<R>* in, double2* out, int64_t n, cudaStream_t s) {
  k_to_c128<R><<<grid_for(n, 256), 256, 0, s>>>(in, out, n);
  CQ_LAUNCHED();
}

template <typename R>
__global__ void k_tq_to_qt(const cplx_t<R>* __restrict__ W, double2* __restrict__ out, int64_t nt,
                           int64_t nq, int64_t ncol, int64_t q0, int64_t nqc) {
  const int64_t total = nqc * nt * ncol;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i % ncol;
    const int64_t t = (i / ncol) % nt;
    const int64_t q = i / (ncol * nt);
    const cplx_t<R> v = W[(t * nq + q0 + q) * ncol + e];
    out[i] = make_double2(v.x, v.y);
  }
}
template <typename R>
void launch_tq_to_qt_c128(const cplx_t<R>* W, double2* out, int64_t nt, int64_t nq, int64_t ncol,
                          int64_t q0, int64_t nqc, cudaStream_t s) {
  k_tq_to_qt<R><<<grid_for(nqc * nt * ncol, 256), 256, 0, s>>>(W, out, nt, nq, ncol, q0, nqc);
  CQ_LAUNCHED();
}

template <typename R>
__global__ void k_qt_to_tq(const double2* __restrict__ in, cplx_t<R>* __restrict__ W, int64_t nt,
                           int64_t nq, int64_t ncol) {
  const int64_t total = nq * nt * ncol;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i % ncol;
    const int64_t q = (i / ncol) % nq;
    const int64_t t = i / (ncol * nq);
    const double2 v = in[(q * nt + t) * ncol + e];
    cplx_t<R> o;
    o.x = (R)v.x;
    o.y = (R)v.y;
    W[i] = o;
  }
}
template <typename R>
void launch_qt_to_tq(const double2* in, cplx_t<R>* W, int64_t nt, int64_t nq, int64_t ncol,
                     cudaStream_t s) {
  k_qt_to_tq<R><<<grid_for(nq * nt * ncol, 256), 256, 0, s>>>(in, W, nt, nq, ncol);
  CQ_LAUNCHED();
}

// ---------------------------------------------------------------------------------------
// Dyson helpers
// ---------------------------------------------------------------------------------------
template <typename R>
__global__ void k_eye_minus(const cplx_t<R>* __restrict__ M, double2* __restrict__ A, int64_t Np,
                            int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i % (Np * Np);
    const cplx_t<R> m = M[i];
    double2 a = make_double2(-(double)m.x, -(double)m.y);
    if (e / Np == e % Np) a.x += 1.0;
    A[i] = a;
  }
}
template <typename R>
void launch_eye_minus(const cplx_t<R>* M, double2* A, int64_t Np, int64_t nprob, cudaStream_t s) {
  const int64_t n = Np * Np * nprob;
  k_eye_minus<R><<<grid_for(n, 256), 256, 0, s>>>(M, A, Np, n);
  CQ_LAUNCHED();
}

template <typename R>
__global__ void k_logdet_trace(const double2* __restrict__ Cf, const cplx_t<R>* __restrict__ M,
                               double* __restrict__ logdet, double2* __restrict__ trace,
                               int64_t Np) {
  const int64_t p = blockIdx.x;
  const double2* c = Cf + p * Np * Np;
  const cplx_t<R>* m = M + p * Np * Np;
  double ld = 0, tr = 0, ti = 0;
  for (int64_t i = threadIdx.x; i < Np; i += blockDim.x) {
    ld += log(c[i * Np + i].x);
    const cplx_t<R> v = m[i * Np + i];
    tr += v.x;
    ti += v.y;
  }
  __shared__ double s0[256], s1[256], s2[256];
  s0[threadIdx.x] = ld;
  s1[threadIdx.x] = tr;
  s2[threadIdx.x] = ti;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s0[threadIdx.x] += s0[threadIdx.x + w];
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    logdet[p] = 2.0 * s0[0];
    trace[p] = make_double2(s1[0], s2[0]);
  }
}
template <typename R>
void launch_logdet_trace(const double2* C, const cplx_t<R>* M, double* logdet, double2* trace,
                         int64_t Np, int64_t nprob, cudaStream_t s) {
  k_logdet_trace<R><<<(unsigned)nprob, 256, 0, s>>>(C, M, logdet, trace, Np);
  CQ_LAUNCHED();
}

// eps[t q] = fac[q] sum_PQ chi_P W_PQ conj(chi_Q) for one (t, q) matrix per CTA: each warp
// takes rows P, its lanes sweep Q (coalesced rows of W), t_P = sum_Q W_PQ conj(chi_Q) is
// formed per lane and multiplied by chi_P once per row; FP64 accumulation.
template <typename R>
__global__ void __launch_bounds__(256) k_eps_head(const cplx_t<R>* __restrict__ W,
                                                  const double2* __restrict__ chi,
                                                  const double* __restrict__ fac,
                                                  double2* __restrict__ eps, int64_t nq,
                                                  int64_t Np) {
  const int64_t tq = blockIdx.x;  // t * nq + q
  const int64_t q = tq % nq;
  const cplx_t<R>* w = W + tq * Np * Np;
  const double2* x = chi + q * Np;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  double ar = 0, ai = 0;
  for (int64_t P = warp; P < Np; P += nwarp) {
    const cplx_t<R>* row = w + P * Np;
    double tr = 0, ti = 0;
#pragma unroll 4
    for (int64_t Q = lane; Q < Np; Q += 32) {
      const cplx_t<R> v = row[Q];
      const double2 b = __ldg(x + Q);
      tr += (double)v.x * b.x + (double)v.y * b.y;  // v conj(b)
      ti += (double)v.y * b.x - (double)v.x * b.y;
    }
    const double2 a = __ldg(x + P);
    ar += a.x * tr - a.y * ti;
    ai += a.x * ti + a.y * tr;
  }
  for (int o = 16; o > 0; o >>= 1) {
    ar += __shfl_down_sync(0xffffffffu, ar, o);
    ai += __shfl_down_sync(0xffffffffu, ai, o);
  }
  __shared__ double s0[8], s1[8];
  if (lane == 0) {
    s0[warp] = ar;
    s1[warp] = ai;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0, i = 0;
    for (int k = 0; k < nwarp; ++k) {
      r += s0[k];
      i += s1[k];
    }
    eps[tq] = make_double2(fac[q] * r, fac[q] * i);
  }
}
template <typename R>
void launch_eps_head(const cplx_t<R>* W, const double2* chi, const double* fac, double2* eps,
                     int64_t nt, int64_t nq, int64_t Np, cudaStream_t s) {
  k_eps_head<R><<<(unsigned)(nt * nq), 256, 0, s>>>(W, chi, fac, eps, nq, Np);
  CQ_LAUNCHED();
}

// ---------------------------------------------------------------------------------------
// generic strided batched complex GEMM on CUDA cores (64x64 tile, 4x4 per thread)
// ---------------------------------------------------------------------------------------
template <typename T> struct CReal;
template <> struct CReal<float2> { using type = float; };
template <> struct CReal<double2> { using type = double; };

template <typename TA, typename TB, typename TC, typename Acc>
__global__ void __launch_bounds__(256) k_gemm_simt(GemmDesc d, const TA* __restrict__ A,
                                                   const TB* __restrict__ B, TC* __restrict__ C) {
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ Acc sAr[BK][BM + 1], sAi[BK][BM + 1], sBr[BK][BN + 1], sBi[BK][BN + 1];
  const int64_t b = blockIdx.z;
  const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
  const TA* Ab = A + b * d.bsa;
  const TB* Bb = B + b * d.bsb;
  TC* Cb = C + b * d.bsc;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  Acc cr[4][4] = {}, ci[4][4] = {};
  const Acc sa = d.conj_a ? -1 : 1, sb = d.conj_b ? -1 : 1;
  for (int64_t k0 = 0; k0 < d.K; k0 += BK) {
    for (int i = threadIdx.x; i < BM * BK; i += 256) {
      const int mm = i % BM, kk = i / BM;
      const int64_t m = m0 + mm, k = k0 + kk;
      Acc vr = 0, vi = 0;
      if (m < d.M && k < d.K) {
        const TA v = Ab[m * d.sam + k * d.sak];
        vr = (Acc)v.x;
        vi = sa * (Acc)v.y;
      }
      sAr[kk][mm] = vr;
      sAi[kk][mm] = vi;
    }
    for (int i = threadIdx.x; i < BN * BK; i += 256) {
      const int nn = i % BN, kk = i / BN;
      const int64_t n = n0 + nn, k = k0 + kk;
      Acc vr = 0, vi = 0;
      if (n < d.N && k < d.K) {
        const TB v = Bb[k * d.sbk + n * d.sbn];
        vr = (Acc)v.x;
        vi = sb * (Acc)v.y;
      }
      sBr[kk][nn] = vr;
      sBi[kk][nn] = vi;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      Acc ar[4], ai[4], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        ar[i] = sAr[kk][ty + 16 * i];
        ai[i] = sAi[kk][ty + 16 * i];
        br[i] = sBr[kk][tx + 16 * i];
        bi[i] = sBi[kk][tx + 16 * i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          cr[i][j] += ar[i] * br[j] - ai[i] * bi[j];
          ci[i][j] += ar[i] * bi[j] + ai[i] * br[j];
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
      if (m < d.M && n < d.N) {
        TC* c = Cb + m * d.scm + n * d.scn;
        double re = d.alpha.x * (double)cr[i][j] - d.alpha.y * (double)ci[i][j];
        double im = d.alpha.x * (double)ci[i][j] + d.alpha.y * (double)cr[i][j];
        if (d.beta.x != 0.0 || d.beta.y != 0.0) {
          const TC o = *c;
          re += d.beta.x * (double)o.x - d.beta.y * (double)o.y;
          im += d.beta.x * (double)o.y + d.beta.y * (double)o.x;
        }
        TC r;
        r.x = re;
        r.y = im;
        *c = r;
      }
    }
}

template <typename TA, typename TB, typename TC, typename Acc>
void launch_gemm_simt(const GemmDesc& d, const TA* A, const TB* B, TC* C, cudaStream_t s) {
  CQ_REQUIRE(d.batch <= 65535, COQUI_B200_EINVAL, "gemm batch too large");
  dim3 grid((unsigned)((d.N + 63) / 64), (unsigned)((d.M + 63) / 64), (unsigned)d.batch);
  k_gemm_simt<TA, TB, TC, Acc><<<grid, 256, 0, s>>>(d, A, B, C);
  CQ_LAUNCHED();
}

// ---------------------------------------------------------------------------------------
// explicit instantiations
// ---------------------------------------------------------------------------------------
#define CQ_INST(R)                                                                                \
  template void launch_pi_fused<R>(const cplx_t<R>*, const cplx_t<R>*, cplx_t<R>*, int64_t,     \
                                   KGrid, double, cudaStream_t);                                \
  template void launch_sigma_fused<R>(const cplx_t<R>*, const cplx_t<R>*, const cplx_t<R>*,    \
                                      cplx_t<R>*, cplx_t<R>*, int64_t, KGrid, cudaStream_t);    \
  template void launch_dft_plain<R>(cplx_t<R>*, int64_t, KGrid, int, double, int64_t, int64_t,  \
                                    cudaStream_t);                                              \
  template void launch_ir_transform<R>(cplx_t<R>*, int64_t, int, int, const double2*,           \
                                       cudaStream_t);                                           \
  template void launch_ir_transform_real<R>(cplx_t<R>*, int64_t, int, int, const double*,       \
                                            cudaStream_t);                                      \
  template void launch_from_c128<R>(const double2*, cplx_t<R>*, int64_t, cudaStream_t);         \
  template void launch_to_c128<R>(const cplx_t<R>*, double2*, int64_t, cudaStream_t);           \
  template void launch_eye_minus<R>(const cplx_t<R>*, double2*, int64_t, int64_t, cudaStream_t); \
  template void launch_logdet_trace<R>(const double2*, const cplx_t<R>*, double*, double2*,     \
                                       int64_t, int64_t, cudaStream_t);                         \
  template void launch_eps_head<R>(const cplx_t<R>*, const double2*, const double*, double2*,   \
                                   int64_t, int64_t, int64_t, cudaStream_t);                    \
  template void launch_tq_to_qt_c128<R>(const cplx_t<R>*, double2*, int64_t, int64_t, int64_t,  \
                                        int64_t, int64_t, cudaStream_t);                        \
  template void launch_qt_to_tq<R>(const double2*, cplx_t<R>*, int64_t, int64_t, int64_t,      \
                                   cudaStream_t);

CQ_INST(float)
CQ_INST(double)

#define CQ_GEMM_INST(TA, TB, TC, ACC)                                                   \
  template void launch_gemm_simt<TA, TB, TC, ACC>(const GemmDesc&, const TA*, const TB*, TC*, \
                                                  cudaStream_t);
CQ_GEMM_INST(float2, float2, float2, float)
CQ_GEMM_INST(float2, double2, float2, float)
CQ_GEMM_INST(double2, float2, float2, float)
CQ_GEMM_INST(double2, double2, float2, float)
CQ_GEMM_INST(float2, float2, double2, double)
CQ_GEMM_INST(float2, double2, double2, double)
CQ_GEMM_INST(double2, float2, double2, double)
CQ_GEMM_INST(double2, double2, double2, double)

void ph_symmetric_matrices(const double* Twt_bb, const double* Ttw_bb, int64_t nt, int64_t nwb,
                           std::vector<double2>& Twt_pos, std::vector<double2>& Ttw_pos) {
  const int64_t nth = (nt + 1) / 2, nwh = (nwb + 1) / 2;
  auto at = [](const double* p, int64_t i) { return make_double2(p[2 * i], p[2 * i + 1]); };
  Twt_pos.assign(nwh * nth, make_double2(0, 0));
  for (int64_t n = 0; n < nwh; ++n)
    for (int64_t it = 0; it < nth; ++it) {
      const int64_t iw = nwb / 2 + n, imt = nt - it - 1;
      double2 v = at(Twt_bb, iw * nt + it);
      if (it != imt) {
        const double2 u = at(Twt_bb, iw * nt + imt);
        v.x += u.x;
        v.y += u.y;
      }
      Twt_pos[n * nth + it] = v;
    }
  Ttw_pos.assign(nth * nwh, make_double2(0, 0));
  for (int64_t it = 0; it < nth; ++it)
    for (int64_t n = 0; n < nwh; ++n) {
      const int64_t iw = nwb / 2 + n, imw = nwb / 2 - n;
      double2 v = at(Ttw_bb, it * nwb + iw);
      if (iw != imw) {
        const double2 u = at(Ttw_bb, it * nwb + imw);
        v.x += u.x;
        v.y += u.y;
      }
      Ttw_pos[it * nwh + n] = v;
    }
}

namespace {
__global__ void k_check_finite(const double2* __restrict__ p, int64_t n, int* __restrict__ flag) {
  bool bad = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = p[i];
    bad |= !isfinite(v.x) || !isfinite(v.y);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(flag, 1);
}
}  // namespace

void launch_check_finite(const double2* p, int64_t n, int* flag, cudaStream_t s) {
  if (n <= 0) return;
  k_check_finite<<<grid_for(n, 256), 256, 0, s>>>(p, n, flag);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

}  // namespace cq
