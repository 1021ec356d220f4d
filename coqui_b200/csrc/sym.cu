// Kernels of the symmetry-reduced (IBZ) k-space path: unfolding of the IBZ Green's function,
// the transposed gather of the IBZ polarizability, and the per-symmetry self-energy sums.
// All three are HBM-bound gathers: one pass over their inputs, coalesced along the
// contiguous matrix or auxiliary-pair index.
#include <algorithm>
#include <type_traits>

#include "sym.cuh"

namespace cq {

// one CTA of 32 x 8 threads per 32 x 32 tile of one (t, k) matrix
__global__ void k_unfold_g(const double2* __restrict__ Gi, double2* __restrict__ G,
                           const int* __restrict__ src, int64_t nk, int64_t nk_ibz, int64_t nb) {
  __shared__ double2 tile[32][33];
  const int64_t tk = blockIdx.z;
  const int64_t t = tk / nk, k = tk % nk;
  const int code = src[k];
  const bool tr = (code >> 30) & 1;
  const int64_t j = code & 0x3fffffff;
  const double2* in = Gi + (t * nk_ibz + j) * nb * nb;
  double2* out = G + tk * nb * nb;
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  if (!tr) {
    for (int dy = threadIdx.y; dy < 32; dy += 8) {
      const int64_t r = r0 + dy, c = c0 + threadIdx.x;
      if (r < nb && c < nb) out[r * nb + c] = in[r * nb + c];
    }
    return;
  }
  // out[r][c] = in[c][r]: read rows c0.. of in, write rows r0.. of out
  for (int dy = threadIdx.y; dy < 32; dy += 8) {
    const int64_t r = c0 + dy, c = r0 + threadIdx.x;  // in[r][c]
    if (r < nb && c < nb) tile[dy][threadIdx.x] = in[r * nb + c];
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += 8) {
    const int64_t r = r0 + dy, c = c0 + threadIdx.x;  // out[r][c] = in[c][r]
    if (r < nb && c < nb) out[r * nb + c] = tile[threadIdx.x][dy];
  }
}

void launch_unfold_g(const double2* Gi, double2* G, const int* src, int64_t nt, int64_t nk,
                     int64_t nk_ibz, int64_t nb, cudaStream_t s) {
  CQ_REQUIRE(nt * nk <= 65535, COQUI_B200_EUNSUPPORTED, "unfold: too many (tau, k) matrices");
  const unsigned nbt = (unsigned)((nb + 31) / 32);
  k_unfold_g<<<dim3(nbt, nbt, (unsigned)(nt * nk)), dim3(32, 8), 0, s>>>(Gi, G, src, nk, nk_ibz,
                                                                          nb);
  count_launch(1);
  CQ_CHECK_CUDA(cudaGetLastError());
}

template <typename R>
__global__ void k_gather_transpose(const cplx_t<R>* __restrict__ in, cplx_t<R>* __restrict__ out,
                                   const int* __restrict__ qsrc, int64_t nq, int64_t nqo,
                                   int64_t Np) {
  __shared__ cplx_t<R> tile[32][33];
  const int64_t ti = blockIdx.z;
  const int64_t t = ti / nqo, i = ti % nqo;
  const cplx_t<R>* a = in + (t * nq + qsrc[i]) * Np * Np;
  cplx_t<R>* b = out + ti * Np * Np;
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  for (int dy = threadIdx.y; dy < 32; dy += 8) {
    const int64_t r = c0 + dy, c = r0 + threadIdx.x;
    if (r < Np && c < Np) tile[dy][threadIdx.x] = a[r * Np + c];
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += 8) {
    const int64_t r = r0 + dy, c = c0 + threadIdx.x;
    if (r < Np && c < Np) b[r * Np + c] = tile[threadIdx.x][dy];
  }
}

template <typename R>
void launch_gather_transpose(const cplx_t<R>* in, cplx_t<R>* out, const int* qsrc, int64_t nt,
                             int64_t nq, int64_t nqo, int64_t Np, cudaStream_t s) {
  CQ_REQUIRE(nt * nqo <= 65535 && Np <= 65535 * 32, COQUI_B200_EUNSUPPORTED,
             "gather: too many (tau, q) matrices");
  const unsigned nbt = (unsigned)((Np + 31) / 32);
  k_gather_transpose<R><<<dim3(nbt, nbt, (unsigned)(nt * nqo)), dim3(32, 8), 0, s>>>(
      in, out, qsrc, nq, nqo, Np);
  count_launch(1);
  CQ_CHECK_CUDA(cudaGetLastError());
}

// One CTA per tile of E consecutive auxiliary pairs: the tile of every G(k) and W(q_ibz) is
// staged in shared memory once, then each (isym, ik) output row of the tile is summed over its
// terms from there (E threads per row, blockDim / E rows at a time).  The sum runs in the
// storage precision: complex64 terms accumulate in FP32 with packed FMAs (converting every
// term to FP64 made the FP32 -> FP64 conversions, not memory, the limit), complex128 in FP64.
template <typename R, int E>
__global__ void __launch_bounds__(256) k_sigma_ksum(const cplx_t<R>* __restrict__ G,
                                                    const cplx_t<R>* __restrict__ W,
                                                    const int4* __restrict__ terms,
                                                    const int2* __restrict__ rows, int nrow,
                                                    int nk, int nqi, int64_t ncol, double factor,
                                                    cplx_t<R>* __restrict__ S) {
  extern __shared__ __align__(16) unsigned char sym_smem[];
  cplx_t<R>* sv = reinterpret_cast<cplx_t<R>*>(sym_smem);  // (nk + nqi) x E: G rows, W rows
  const int64_t e0 = (int64_t)blockIdx.x * E;
  const int ne = (int)((ncol - e0) < E ? (ncol - e0) : E);
  for (int i = threadIdx.x; i < (nk + nqi) * E; i += blockDim.x) {
    const int r = i / E, e = i % E;
    cplx_t<R> v;
    v.x = 0;
    v.y = 0;
    if (e < ne) v = (r < nk) ? G[(int64_t)r * ncol + e0 + e] : W[(int64_t)(r - nk) * ncol + e0 + e];
    sv[i] = v;
  }
  __syncthreads();
  const cplx_t<R>* sW = sv + nk * E;
  const int e = threadIdx.x % E;
  for (int p = threadIdx.x / E; p < nrow; p += blockDim.x / E) {
    const int2 rw = rows[p];  // (first term, term count)
    cplx_t<R> acc;
    acc.x = 0;
    acc.y = 0;
    for (int j = 0; j < rw.y; ++j) {
      const int4 tj = terms[rw.x + j];
      cplx_t<R> g = sv[tj.y * E + e];
      cplx_t<R> w = sW[tj.x * E + e];
      if (tj.z & 1) g.y = -g.y;
      if (tj.z & 2) w.y = -w.y;
      if constexpr (std::is_same<R, float>::value) {
        // (re, im) += g * w as two packed FP32 FMAs (sm_100)
        acc = __ffma2_rn(make_float2(g.x, g.x), w, acc);
        acc = __ffma2_rn(make_float2(-g.y, g.y), make_float2(w.y, w.x), acc);
      } else {
        acc.x = fma(g.x, w.x, fma(-g.y, w.y, acc.x));
        acc.y = fma(g.x, w.y, fma(g.y, w.x, acc.y));
      }
    }
    if (e < ne) {
      cplx_t<R> o;
      o.x = (R)(factor * acc.x);
      o.y = (R)(factor * acc.y);
      S[(int64_t)p * ncol + e0 + e] = o;
    }
  }
}

template <typename R, int E>
static void ksum_launch(const cplx_t<R>* G, const cplx_t<R>* W, const int4* terms,
                        const int2* rows, int nrow, int nk, int nqi, int64_t ncol,
                        double factor, cplx_t<R>* S, size_t smem, cudaStream_t s) {
  CQ_CHECK_CUDA(cudaFuncSetAttribute(k_sigma_ksum<R, E>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t nblk = (ncol + E - 1) / E;
  CQ_REQUIRE(nblk <= 0x7fffffff, COQUI_B200_EUNSUPPORTED, "sigma k-sum: too many columns");
  k_sigma_ksum<R, E><<<(unsigned)nblk, 256, smem, s>>>(G, W, terms, rows, nrow, nk, nqi, ncol,
                                                      factor, S);
}

template <typename R>
void launch_sigma_ksum(const cplx_t<R>* G, const cplx_t<R>* W, const int4* terms,
                       const int2* rows, int64_t nrow, int64_t nk, int64_t nqi, int64_t ncol,
                       double factor, cplx_t<R>* S, cudaStream_t s) {
  const size_t per = (size_t)(nk + nqi) * sizeof(cplx_t<R>);
  const size_t cap = 160 * 1024;
  CQ_REQUIRE(per <= cap && nrow <= 0x7fffffff, COQUI_B200_EUNSUPPORTED,
             "sigma k-sum: too many k-points for one shared-memory tile");
  if (per * 32 <= cap)
    ksum_launch<R, 32>(G, W, terms, rows, (int)nrow, (int)nk, (int)nqi, ncol, factor, S, per * 32, s);
  else if (per * 16 <= cap)
    ksum_launch<R, 16>(G, W, terms, rows, (int)nrow, (int)nk, (int)nqi, ncol, factor, S, per * 16, s);
  else if (per * 8 <= cap)
    ksum_launch<R, 8>(G, W, terms, rows, (int)nrow, (int)nk, (int)nqi, ncol, factor, S, per * 8, s);
  else
    ksum_launch<R, 1>(G, W, terms, rows, (int)nrow, (int)nk, (int)nqi, ncol, factor, S, per, s);
  count_launch(1);
  CQ_CHECK_CUDA(cudaGetLastError());
}

// out[i] += sum_s R[s * n + i]
__global__ void k_add_blocks(const double2* __restrict__ Rb, double2* __restrict__ out,
                             int64_t nblk, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double2 a = out[i];
    for (int64_t b = 0; b < nblk; ++b) {
      const double2 v = Rb[b * n + i];
      a.x += v.x;
      a.y += v.y;
    }
    out[i] = a;
  }
}

void launch_add_blocks(const double2* Rb, double2* out, int64_t nblk, int64_t n, cudaStream_t s) {
  k_add_blocks<<<grid_for(n, 256), 256, 0, s>>>(Rb, out, nblk, n);
  count_launch(1);
  CQ_CHECK_CUDA(cudaGetLastError());
}

#define CQ_SYM_INST(R)                                                                        \
  template void launch_gather_transpose<R>(const cplx_t<R>*, cplx_t<R>*, const int*, int64_t, \
                                           int64_t, int64_t, int64_t, cudaStream_t);          \
  template void launch_sigma_ksum<R>(const cplx_t<R>*, const cplx_t<R>*, const int4*,         \
                                     const int2*, int64_t, int64_t, int64_t, int64_t, double,  \
                                     cplx_t<R>*, cudaStream_t);

CQ_SYM_INST(float)
CQ_SYM_INST(double)

}  // namespace cq
