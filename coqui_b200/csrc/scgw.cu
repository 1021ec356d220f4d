// Device pieces of the self-consistent GW loop: Dyson equation for G on the fermionic
// Matsubara grid (simple_dyson.cpp:66-77), Hermitian symmetrisation (scf_common.hpp:70-86),
// trace products for the energies (scf_common.cpp:44-136) and the vector algebra of damping
// (damp_t.hpp:34-48) and commutator DIIS (diis_alg.hpp, vspace_fock_sigma.hpp).
#include <algorithm>
#include <vector>

#include "scgw.cuh"

namespace cq {

namespace {

constexpr int kGjMaxN = 96;  // Gauss-Jordan in shared memory up to 96 x 96 complex128

__device__ __forceinline__ double2 cmul2(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void k_hermitize(double2* __restrict__ A, int64_t nb, int64_t nmat) {
  const int64_t per = nb * nb;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < per * nmat;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = idx / per, e = idx % per;
    const int64_t i = e / nb, j = e % nb;
    if (i > j) continue;  // the thread of (i <= j) writes both entries
    double2* a = A + m * per;
    const double2 x = a[i * nb + j], y = a[j * nb + i];
    // (A + A^H)/2: entry (i, j) = (x + conj(y))/2, entry (j, i) its conjugate
    const double2 v = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
    a[i * nb + j] = v;
    if (i != j) a[j * nb + i] = make_double2(v.x, -v.y);
  }
}

__global__ void __launch_bounds__(256) k_trace_products(const double2* __restrict__ A,
                                                        const double2* __restrict__ B,
                                                        double2* __restrict__ out, int64_t nb,
                                                        int64_t b_mod) {
  __shared__ double red[2][256];
  const int64_t m = blockIdx.x;
  const int64_t bm = b_mod ? m % b_mod : m;
  const double2* a = A + m * nb * nb;
  const double2* b = B + bm * nb * nb;
  double sr = 0, si = 0;
  for (int64_t e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int64_t i = e / nb, j = e % nb;
    const double2 p = cmul2(a[e], b[j * nb + i]);
    sr += p.x;
    si += p.y;
  }
  red[0][threadIdx.x] = sr;
  red[1][threadIdx.x] = si;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      red[0][threadIdx.x] += red[0][threadIdx.x + w];
      red[1][threadIdx.x] += red[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[m] = make_double2(red[0][0], red[1][0]);
}

__global__ void k_build_x(const double2* __restrict__ S, const double2* __restrict__ H0,
                          const double2* __restrict__ F, const double2* __restrict__ Sw,
                          double2* __restrict__ X, const int64_t* __restrict__ wn, double beta,
                          double mu, int64_t nw, int64_t nk, int64_t nb) {
  const int64_t per_k = nb * nb, total = nw * nk * per_k;
  const double pi = 3.14159265358979323846;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t w = idx / (nk * per_k);
    const int64_t ke = idx % (nk * per_k);
    const double om = pi * (double)wn[w] / beta;  // i omega_n + mu = (mu, om)
    const double2 s = S[ke], h = H0[ke], f = F[ke], sg = Sw[idx];
    X[idx] = make_double2(mu * s.x - om * s.y - h.x - f.x - sg.x,
                          mu * s.y + om * s.x - h.y - f.y - sg.y);
  }
}

// In-place Gauss-Jordan inverse with partial (row) pivoting; the row swaps are undone on the
// columns at the end.  One CTA per matrix.
__global__ void __launch_bounds__(256) k_gauss_jordan(double2* __restrict__ Aall, int n,
                                                      int* __restrict__ info) {
  extern __shared__ __align__(16) unsigned char gj_raw[];
  double2* A = reinterpret_cast<double2*>(gj_raw);
  double2* col = A + n * n;
  __shared__ int s_perm[kGjMaxN];
  __shared__ int s_piv;
  __shared__ int s_bad;
  double2* g = Aall + (int64_t)blockIdx.x * n * n;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) A[e] = g[e];
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = 0; k < n; ++k) {
    if (warp == 0) {
      double best = -1.0;
      int bi = k;
      for (int i = k + lane; i < n; i += 32) {
        const double2 v = A[i * n + k];
        const double m = v.x * v.x + v.y * v.y;
        if (m > best) {
          best = m;
          bi = i;
        }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (lane == 0) {
        s_piv = bi;
        s_perm[k] = bi;
        if (!(best > 0.0)) s_bad = 1;
      }
    }
    __syncthreads();
    const int pr = s_piv;
    if (pr != k)
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double2 t = A[k * n + j];
        A[k * n + j] = A[pr * n + j];
        A[pr * n + j] = t;
      }
    __syncthreads();
    double2 piv = A[k * n + k];
    const double pm = piv.x * piv.x + piv.y * piv.y;
    const double2 inv = pm > 0.0 ? make_double2(piv.x / pm, -piv.y / pm) : make_double2(1.0, 0.0);
    for (int i = threadIdx.x; i < n; i += blockDim.x) col[i] = A[i * n + k];
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x)
      A[k * n + j] = (j == k) ? inv : cmul2(A[k * n + j], inv);
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      if (i == k) continue;
      const double2 f = col[i];
      const double2 base = (j == k) ? make_double2(0.0, 0.0) : A[e];
      const double2 p = cmul2(A[k * n + j], f);
      A[e] = make_double2(base.x - p.x, base.y - p.y);
    }
    __syncthreads();
  }
  for (int k = n - 1; k >= 0; --k) {
    const int pk = s_perm[k];
    if (pk != k)
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double2 t = A[i * n + k];
        A[i * n + k] = A[i * n + pk];
        A[i * n + pk] = t;
      }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) g[e] = A[e];
  if (threadIdx.x == 0) info[blockIdx.x] = s_bad;
}

__global__ void k_axpby(const double2* __restrict__ x, double2* __restrict__ y, double a, double b,
                        int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 u = x[i], v = y[i];
    y[i] = make_double2(a * u.x + b * v.x, a * u.y + b * v.y);
  }
}

__global__ void k_axpy(const double2* __restrict__ x, double2* __restrict__ y, double2 c, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 p = cmul2(c, x[i]);
    y[i].x += p.x;
    y[i].y += p.y;
  }
}

__global__ void k_extract_diag(const double2* __restrict__ A, double2* __restrict__ out, int64_t nb,
                               int64_t nmat) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb * nmat;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = i / nb, d = i % nb;
    out[i] = A[m * nb * nb + d * nb + d];
  }
}

__global__ void k_add_diag(double2* __restrict__ A, const double2* __restrict__ dv, int64_t nb,
                           int64_t nmat) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb * nmat;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = i / nb, d = i % nb;
    double2& a = A[m * nb * nb + d * nb + d];
    a.x += dv[i].x;
    a.y += dv[i].y;
  }
}

constexpr int kRedBlocks = 592;

__global__ void __launch_bounds__(256) k_maxabs_diff(const double2* __restrict__ a,
                                                     const double2* __restrict__ b, int64_t n,
                                                     double* __restrict__ part) {
  __shared__ double red[256];
  double m = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double2 d = a[i];
    if (b) {
      d.x -= b[i].x;
      d.y -= b[i].y;
    }
    m = fmax(m, d.x * d.x + d.y * d.y);
  }
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(256) k_dotc(const double2* __restrict__ a,
                                              const double2* __restrict__ b, int64_t n,
                                              double* __restrict__ part) {
  __shared__ double red[2][256];
  double sr = 0, si = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 u = a[i], v = b[i];  // conj(u) v
    sr += u.x * v.x + u.y * v.y;
    si += u.x * v.y - u.y * v.x;
  }
  red[0][threadIdx.x] = sr;
  red[1][threadIdx.x] = si;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      red[0][threadIdx.x] += red[0][threadIdx.x + w];
      red[1][threadIdx.x] += red[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = red[0][0];
    part[2 * blockIdx.x + 1] = red[1][0];
  }
}

// rho[Q] = scale sum_k sum_b T[k, Q, b] conj(X[k, Q, b]): one warp per Q, FP64
__global__ void __launch_bounds__(256) k_aux_diag(const double2* __restrict__ T,
                                                  const double2* __restrict__ X,
                                                  double2* __restrict__ rho, int64_t nk,
                                                  int64_t Np, int64_t nb, double scale) {
  const int64_t Q = (int64_t)blockIdx.x * 8 + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (Q >= Np) return;
  double sr = 0, si = 0;
  for (int64_t k = 0; k < nk; ++k) {
    const double2* t = T + (k * Np + Q) * nb;
    const double2* x = X + (k * Np + Q) * nb;
    for (int64_t b = lane; b < nb; b += 32) {
      const double2 a = t[b], y = x[b];
      sr += a.x * y.x + a.y * y.y;
      si += a.y * y.x - a.x * y.y;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_down_sync(0xffffffffu, sr, o);
    si += __shfl_down_sync(0xffffffffu, si, o);
  }
  if (lane == 0) rho[Q] = make_double2(scale * sr, scale * si);
}

// Y[k, P, b] = d[P] X[k, P, b]
__global__ void k_scale_rows(const double2* __restrict__ X, const double2* __restrict__ d,
                             double2* __restrict__ Y, int64_t nk, int64_t Np, int64_t nb) {
  const int64_t n = nk * Np * nb;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    Y[i] = cmul2(d[(i / nb) % Np], X[i]);
}

// A[s * per + e] *= f[s]
__global__ void k_scale_slices(double2* __restrict__ A, const double* __restrict__ f,
                               int64_t nslice, int64_t per) {
  const int64_t n = nslice * per;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double v = f[i / per];
    A[i] = make_double2(v * A[i].x, v * A[i].y);
  }
}

}  // namespace

void scale_slices(double2* A, const double* f, int64_t nslice, int64_t per, cudaStream_t s) {
  k_scale_slices<<<grid_for(nslice * per, 256), 256, 0, s>>>(A, f, nslice, per);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void aux_diag(const double2* T, const double2* X, double2* rho, int64_t nk, int64_t Np,
              int64_t nb, double scale, cudaStream_t s) {
  k_aux_diag<<<(unsigned)((Np + 7) / 8), 256, 0, s>>>(T, X, rho, nk, Np, nb, scale);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void scale_rows(const double2* X, const double2* d, double2* Y, int64_t nk, int64_t Np,
                int64_t nb, cudaStream_t s) {
  k_scale_rows<<<grid_for(nk * Np * nb, 256), 256, 0, s>>>(X, d, Y, nk, Np, nb);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void hermitize_c128(double2* A, int64_t nb, int64_t nmat, cudaStream_t s) {
  const int64_t n = nb * nb * nmat;
  k_hermitize<<<grid_for(n, 256), 256, 0, s>>>(A, nb, nmat);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void trace_products(const double2* A, const double2* B, double2* out, int64_t nb, int64_t nmat,
                    int64_t b_mod, cudaStream_t s) {
  CQ_REQUIRE(nmat <= 2147483647, COQUI_B200_EINVAL, "trace_products: too many matrices");
  k_trace_products<<<(unsigned)nmat, 256, 0, s>>>(A, B, out, nb, b_mod);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void build_dyson_matrix(const double2* S, const double2* H0, const double2* F,
                        const double2* Sigma_w, double2* X, const int64_t* wn, double beta,
                        double mu, int64_t nw, int64_t nk, int64_t nb, cudaStream_t s) {
  const int64_t n = nw * nk * nb * nb;
  k_build_x<<<grid_for(n, 256), 256, 0, s>>>(S, H0, F, Sigma_w, X, wn, beta, mu, nw, nk, nb);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void invert_batched(double2* A, int64_t nb, int64_t nmat, int* info, cudaStream_t s) {
  CQ_REQUIRE(nb >= 1 && nb <= kGjMaxN, COQUI_B200_EUNSUPPORTED,
             "Dyson equation for G supports at most 96 orbitals");
  CQ_REQUIRE(nmat <= 2147483647, COQUI_B200_EINVAL, "invert_batched: too many matrices");
  const size_t smem = (size_t)(nb * nb + nb) * sizeof(double2);
  static bool set = false;
  if (!set) {
    CQ_CHECK_CUDA(cudaFuncSetAttribute(k_gauss_jordan, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)((kGjMaxN * kGjMaxN + kGjMaxN) * sizeof(double2))));
    set = true;
  }
  k_gauss_jordan<<<(unsigned)nmat, 256, smem, s>>>(A, (int)nb, info);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void extract_diag(const double2* A, double2* out, int64_t nb, int64_t nmat, cudaStream_t s) {
  k_extract_diag<<<grid_for(nb * nmat, 256), 256, 0, s>>>(A, out, nb, nmat);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void add_diag(double2* A, const double2* d, int64_t nb, int64_t nmat, cudaStream_t s) {
  k_add_diag<<<grid_for(nb * nmat, 256), 256, 0, s>>>(A, d, nb, nmat);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void axpby_c128(const double2* x, double2* y, double a, double b, int64_t n, cudaStream_t s) {
  k_axpby<<<grid_for(n, 256), 256, 0, s>>>(x, y, a, b, n);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void axpy_c128(const double2* x, double2* y, double2 c, int64_t n, cudaStream_t s) {
  k_axpy<<<grid_for(n, 256), 256, 0, s>>>(x, y, c, n);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

double maxabs_diff(const double2* a, const double2* b, int64_t n, DevBuf<double>& part,
                   cudaStream_t s) {
  part.ensure(2 * kRedBlocks);
  k_maxabs_diff<<<kRedBlocks, 256, 0, s>>>(a, b, n, part.p);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  std::vector<double> h(kRedBlocks);
  CQ_CHECK_CUDA(cudaMemcpyAsync(h.data(), part.p, kRedBlocks * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
  CQ_CHECK_CUDA(cudaStreamSynchronize(s));
  double m = 0.0;
  for (double v : h) m = std::max(m, v);
  return std::sqrt(m);
}

std::complex<double> dotc(const double2* a, const double2* b, int64_t n, DevBuf<double>& part,
                          cudaStream_t s) {
  part.ensure(2 * kRedBlocks);
  k_dotc<<<kRedBlocks, 256, 0, s>>>(a, b, n, part.p);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  std::vector<double> h(2 * kRedBlocks);
  CQ_CHECK_CUDA(cudaMemcpyAsync(h.data(), part.p, 2 * kRedBlocks * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
  CQ_CHECK_CUDA(cudaStreamSynchronize(s));
  std::complex<double> r = 0.0;
  for (int i = 0; i < kRedBlocks; ++i) r += std::complex<double>(h[2 * i], h[2 * i + 1]);
  return r;
}

void sym_eigen(const std::vector<double>& A, int64_t n, std::vector<double>& ev,
               std::vector<double>& U) {
  std::vector<double> a(A);
  U.assign(n * n, 0.0);
  for (int64_t i = 0; i < n; ++i) U[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0, tot = 0;
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = 0; j < n; ++j) {
        tot += a[i * n + j] * a[i * n + j];
        if (i != j) off += a[i * n + j] * a[i * n + j];
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int64_t p = 0; p < n; ++p)
      for (int64_t q = p + 1; q < n; ++q) {
        const double apq = a[p * n + q];
        if (apq == 0.0) continue;
        // rotation annihilating a_pq (Golub & Van Loan, symmetric Schur decomposition)
        const double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int64_t k = 0; k < n; ++k) {  // A <- A J (columns p, q)
          const double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = cs * akp - sn * akq;
          a[k * n + q] = sn * akp + cs * akq;
        }
        for (int64_t k = 0; k < n; ++k) {  // A <- J^T A (rows p, q)
          const double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = cs * apk - sn * aqk;
          a[q * n + k] = sn * apk + cs * aqk;
        }
        for (int64_t k = 0; k < n; ++k) {  // U <- U J
          const double ukp = U[k * n + p], ukq = U[k * n + q];
          U[k * n + p] = cs * ukp - sn * ukq;
          U[k * n + q] = sn * ukp + cs * ukq;
        }
      }
  }
  ev.resize(n);
  for (int64_t i = 0; i < n; ++i) ev[i] = a[i * n + i];
}

}  // namespace cq
