// Multilayer perceptron of the learned self-energy update: forward, backward and Adam as
// hand-written kernels.  Weights are BF16 in the forward pass (FP32 master copies for the
// optimiser); every product accumulates in FP32.
//
//   z1 = x W1^T + b1, h1 = tanh(z1); z2 = h1 W2^T + b2, h2 = tanh(z2); y = h2 W3^T + b3
//   loss = mean over the batch and outputs of (y - t)^2
#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <vector>

#include "mlp.cuh"

namespace cq {

namespace {

constexpr int TM = 64, TN = 64, TK = 16;  // output tile and K step of the SIMT GEMM

template <typename T> __device__ __forceinline__ float ld(const T* p, int64_t i);
template <> __device__ __forceinline__ float ld<float>(const float* p, int64_t i) { return p[i]; }
template <> __device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p, int64_t i) {
  return __bfloat162float(p[i]);
}

enum Epi { kStore = 0, kBias = 1, kBiasTanh = 2, kTanhGrad = 3 };

// C[m][n] = sum_k A(m, k) B(k, n) with A(m, k) = A[m sam + k sak], B(k, n) = B[k sbk + n sbn];
// epilogue: kBias adds bias[n], kBiasTanh also applies tanh, kTanhGrad multiplies by
// (1 - aux[m][n]^2) (backward through tanh).  256 threads, 4 x 4 outputs per thread.
template <typename TB, int EPI>
__global__ void __launch_bounds__(256) k_gemm(const float* __restrict__ A, int64_t sam, int64_t sak,
                                              const TB* __restrict__ B, int64_t sbk, int64_t sbn,
                                              float* __restrict__ C, int64_t ldc, int64_t M,
                                              int64_t N, int64_t K, const TB* __restrict__ bias,
                                              const float* __restrict__ aux) {
  __shared__ float As[TK][TM + 4];
  __shared__ float Bs[TK][TN + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int64_t m0 = (int64_t)blockIdx.y * TM, n0 = (int64_t)blockIdx.x * TN;
  float acc[4][4] = {};
  for (int64_t k0 = 0; k0 < K; k0 += TK) {
    for (int i = threadIdx.x; i < TM * TK; i += 256) {
      const int mm = i / TK, kk = i % TK;
      const int64_t m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? A[m * sam + k * sak] : 0.f;
    }
    for (int i = threadIdx.x; i < TN * TK; i += 256) {
      const int kk = i / TN, nn = i % TN;
      const int64_t n = n0 + nn, k = k0 + kk;
      Bs[kk][nn] = (n < N && k < K) ? ld<TB>(B, k * sbk + n * sbn) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
      if (m >= M || n >= N) continue;
      float v = acc[i][j];
      if (EPI == kBias || EPI == kBiasTanh) v += ld<TB>(bias, n);
      if (EPI == kBiasTanh) v = tanhf(v);
      if (EPI == kTanhGrad) {
        const float h = aux[m * ldc + n];
        v *= 1.f - h * h;
      }
      C[m * ldc + n] = v;
    }
}

template <typename TB, int EPI>
void gemm(const float* A, int64_t sam, int64_t sak, const TB* B, int64_t sbk, int64_t sbn, float* C,
          int64_t ldc, int64_t M, int64_t N, int64_t K, const TB* bias, const float* aux,
          cudaStream_t s) {
  const dim3 grid((unsigned)((N + TN - 1) / TN), (unsigned)((M + TM - 1) / TM));
  k_gemm<TB, EPI><<<grid, 256, 0, s>>>(A, sam, sak, B, sbk, sbn, C, ldc, M, N, K, bias, aux);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

// out[c] = sum_r A[r][c] (bias gradients), one block per column
__global__ void k_colsum(const float* __restrict__ A, int64_t rows, int64_t cols,
                         float* __restrict__ out) {
  __shared__ float red[256];
  const int64_t c = blockIdx.x;
  float sum = 0.f;
  for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) sum += A[r * cols + c];
  red[threadIdx.x] = sum;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[c] = red[0];
}

// dy = 2 (y - t) / n and per-block partial sums of (y - t)^2
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ dy,
                      int64_t n, float* __restrict__ part) {
  __shared__ float red[256];
  float sum = 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    dy[i] = 2.f * d / (float)n;
    sum += d * d;
  }
  red[threadIdx.x] = sum;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wb,
                       const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr, float c1, float c2) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16(wi);
  }
}

__global__ void k_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    wb[i] = __float2bfloat16(w[i]);
}

__global__ void k_gather_rows(const float* __restrict__ src, const int64_t* __restrict__ idx,
                              float* __restrict__ dst, int64_t rows, int64_t cols) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows * cols;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / cols, c = i % cols;
    dst[i] = src[idx[r] * cols + c];
  }
}

// features (d1/d2, d2/d3) of each sequence, clamped to [-4, 4]; valid flag where the
// differences are resolved
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 csub2(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

__global__ void k_extrap_features(const double2* __restrict__ h, int64_t nel, float* __restrict__ X,
                                  unsigned char* __restrict__ ok) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel;
       e += (int64_t)gridDim.x * blockDim.x) {
    const double2 s0 = h[e], s1 = h[nel + e], s2 = h[2 * nel + e], s3 = h[3 * nel + e];
    const double2 d1 = csub2(s3, s2), d2 = csub2(s2, s1), d3 = csub2(s1, s0);
    const double a1 = hypot(d1.x, d1.y), a2 = hypot(d2.x, d2.y), a3 = hypot(d3.x, d3.y);
    const double scale = fmax(fmax(hypot(s3.x, s3.y), 1e-300), 1e-300);
    const bool valid = a1 > 1e-14 * scale && a2 > 1e-14 * scale && a3 > 1e-14 * scale;
    ok[e] = valid ? 1 : 0;
    double2 q1 = make_double2(0, 0), q2 = make_double2(0, 0);
    if (valid) {
      q1 = cdiv(d1, d2);
      q2 = cdiv(d2, d3);
    }
    X[4 * e + 0] = (float)fmin(4.0, fmax(-4.0, q1.x));
    X[4 * e + 1] = (float)fmin(4.0, fmax(-4.0, q1.y));
    X[4 * e + 2] = (float)fmin(4.0, fmax(-4.0, q2.x));
    X[4 * e + 3] = (float)fmin(4.0, fmax(-4.0, q2.y));
  }
}

__global__ void k_extrap_apply(const double2* __restrict__ h, int64_t nel, const float* __restrict__ Y,
                               const unsigned char* __restrict__ ok, double max_jump,
                               double2* __restrict__ delta) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel;
       e += (int64_t)gridDim.x * blockDim.x) {
    double2 d = make_double2(0, 0);
    if (ok[e]) {
      const double2 d1 = csub2(h[3 * nel + e], h[2 * nel + e]);
      const double yr = Y[2 * e], yi = Y[2 * e + 1];
      d = make_double2(d1.x * yr - d1.y * yi, d1.x * yi + d1.y * yr);
      const double lim = max_jump * hypot(d1.x, d1.y), a = hypot(d.x, d.y);
      if (a > lim) {
        d.x *= lim / a;
        d.y *= lim / a;
      }
    }
    delta[e] = d;
  }
}

void ensure_batch(Mlp& n, int64_t B) {
  if (B <= n.cap) return;
  n.x.ensure(B * n.din);
  n.t.ensure(B * n.dout);
  n.h1.ensure(B * n.width);
  n.h2.ensure(B * n.width);
  n.y.ensure(B * n.dout);
  n.dy.ensure(B * n.dout);
  n.dh2.ensure(B * n.width);
  n.dh1.ensure(B * n.width);
  n.cap = B;
}

}  // namespace

void mlp_init(Mlp& n, int64_t din, int64_t width, int64_t dout, uint64_t seed, cudaStream_t s) {
  n.din = din;
  n.width = width;
  n.dout = dout;
  n.st = s;
  n.nparam = n.ob3() + dout;
  std::vector<float> h(n.nparam, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int64_t off, int64_t rows, int64_t cols) {  // uniform(-a, a), a = sqrt(6/(fan_in+fan_out))
    const double a = std::sqrt(6.0 / (double)(rows + cols));
    std::uniform_real_distribution<double> u(-a, a);
    for (int64_t i = 0; i < rows * cols; ++i) h[off + i] = (float)u(rng);
  };
  fill(n.oW1(), width, din);
  fill(n.oW2(), width, width);
  fill(n.oW3(), dout, width);
  n.w.ensure(n.nparam);
  n.wb.ensure(n.nparam);
  n.g.ensure(n.nparam);
  n.m.ensure(n.nparam);
  n.v.ensure(n.nparam);
  CQ_CHECK_CUDA(cudaMemsetAsync(n.m.p, 0, n.nparam * sizeof(float), s));
  CQ_CHECK_CUDA(cudaMemsetAsync(n.v.p, 0, n.nparam * sizeof(float), s));
  n.adam_t = 0;
  mlp_set_params(n, h.data(), s);
}

void mlp_set_params(Mlp& n, const float* host, cudaStream_t s) {
  CQ_CHECK_CUDA(cudaMemcpyAsync(n.w.p, host, n.nparam * sizeof(float), cudaMemcpyHostToDevice, s));
  k_to_bf16<<<grid_for(n.nparam, 256), 256, 0, s>>>(n.w.p, n.wb.p, n.nparam);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void mlp_forward(Mlp& n, const float* x, int64_t B, float* y, cudaStream_t s) {
  ensure_batch(n, B);
  const __nv_bfloat16* W = n.wb.p;
  const int64_t H = n.width;
  gemm<__nv_bfloat16, kBiasTanh>(x, n.din, 1, W + n.oW1(), 1, n.din, n.h1.p, H, B, H, n.din,
                                 W + n.ob1(), nullptr, s);
  gemm<__nv_bfloat16, kBiasTanh>(n.h1.p, H, 1, W + n.oW2(), 1, H, n.h2.p, H, B, H, H,
                                 W + n.ob2(), nullptr, s);
  gemm<__nv_bfloat16, kBias>(n.h2.p, H, 1, W + n.oW3(), 1, H, y, n.dout, B, n.dout, H,
                             W + n.ob3(), nullptr, s);
}

float mlp_backward(Mlp& n, const float* x, const float* t, int64_t B, cudaStream_t s) {
  ensure_batch(n, B);
  const int64_t H = n.width, D = n.dout, nout = B * D;
  mlp_forward(n, x, B, n.y.p, s);
  const int nblk = 148;
  n.part.ensure(nblk);
  k_mse<<<nblk, 256, 0, s>>>(n.y.p, t, n.dy.p, nout, n.part.p);
  count_launch();
  float* g = n.g.p;
  const __nv_bfloat16* W = n.wb.p;
  // output layer: dW3 = dy^T h2, db3 = colsum(dy)
  gemm<float, kStore>(n.dy.p, 1, D, n.h2.p, H, 1, g + n.oW3(), H, D, H, B, nullptr, nullptr, s);
  k_colsum<<<(unsigned)D, 256, 0, s>>>(n.dy.p, B, D, g + n.ob3());
  count_launch();
  // dz2 = (dy W3) * (1 - h2^2)
  gemm<__nv_bfloat16, kTanhGrad>(n.dy.p, D, 1, W + n.oW3(), H, 1, n.dh2.p, H, B, H, D, nullptr,
                                 n.h2.p, s);
  gemm<float, kStore>(n.dh2.p, 1, H, n.h1.p, H, 1, g + n.oW2(), H, H, H, B, nullptr, nullptr, s);
  k_colsum<<<(unsigned)H, 256, 0, s>>>(n.dh2.p, B, H, g + n.ob2());
  count_launch();
  // dz1 = (dz2 W2) * (1 - h1^2)
  gemm<__nv_bfloat16, kTanhGrad>(n.dh2.p, H, 1, W + n.oW2(), H, 1, n.dh1.p, H, B, H, H, nullptr,
                                 n.h1.p, s);
  gemm<float, kStore>(n.dh1.p, 1, H, x, n.din, 1, g + n.oW1(), n.din, H, n.din, B, nullptr,
                      nullptr, s);
  k_colsum<<<(unsigned)H, 256, 0, s>>>(n.dh1.p, B, H, g + n.ob1());
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  std::vector<float> part(nblk);
  CQ_CHECK_CUDA(cudaMemcpyAsync(part.data(), n.part.p, nblk * sizeof(float), cudaMemcpyDeviceToHost, s));
  CQ_CHECK_CUDA(cudaStreamSynchronize(s));
  double sum = 0;
  for (float v : part) sum += v;
  return (float)(sum / (double)nout);
}

void mlp_extrapolate(Mlp& n, const double2* hist, int64_t nel, double max_jump, double2* delta,
                     cudaStream_t s) {
  CQ_REQUIRE(n.din == 4 && n.dout == 2, COQUI_B200_EINVAL,
             "the extrapolating network takes 4 inputs and gives 2 outputs");
  DevBuf<float> X, Y;
  DevBuf<unsigned char> ok;
  X.ensure(nel * 4);
  Y.ensure(nel * 2);
  ok.ensure(nel);
  k_extrap_features<<<grid_for(nel, 256), 256, 0, s>>>(hist, nel, X.p, ok.p);
  count_launch();
  mlp_forward(n, X.p, nel, Y.p, s);
  k_extrap_apply<<<grid_for(nel, 256), 256, 0, s>>>(hist, nel, Y.p, ok.p, max_jump, delta);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  CQ_CHECK_CUDA(cudaStreamSynchronize(s));  // X, Y, ok are freed on return
}

void mlp_adam_step(Mlp& n, float lr, cudaStream_t s) {
  ++n.adam_t;
  const float c1 = 1.f - std::pow(0.9f, (float)n.adam_t);
  const float c2 = 1.f - std::pow(0.999f, (float)n.adam_t);
  k_adam<<<grid_for(n.nparam, 256), 256, 0, s>>>(n.w.p, n.wb.p, n.g.p, n.m.p, n.v.p, n.nparam, lr,
                                                 c1, c2);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

}  // namespace cq

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
struct coqui_b200_mlp {
  cq::Mlp net;
  std::string err;
};

cq::Mlp& mlp_net(coqui_b200_mlp* h) { return h->net; }

namespace {
template <typename F> int mlp_guarded(coqui_b200_mlp* h, F&& f) {
  if (!h) return COQUI_B200_EINVAL;
  try {
    CQ_CHECK_CUDA(cudaSetDevice(h->net.dev));
    f();
    CQ_CHECK_CUDA(cudaStreamSynchronize(h->net.st));
    h->err.clear();
    return COQUI_B200_OK;
  } catch (const cq::Error& e) {
    h->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    h->err = e.what();
    return COQUI_B200_EINVAL;
  }
}
}  // namespace

extern "C" {

int coqui_b200_mlp_create(coqui_b200_mlp** out, int64_t in_dim, int64_t width, int64_t out_dim,
                          uint64_t seed, int device) {
  if (!out || in_dim < 1 || width < 1 || out_dim < 1) return COQUI_B200_EINVAL;
  *out = nullptr;
  auto* h = new (std::nothrow) coqui_b200_mlp();
  if (!h) return COQUI_B200_ENOMEM;
  h->net.dev = device;
  int rc = mlp_guarded(h, [&] {
    CQ_CHECK_CUDA(cudaStreamCreateWithFlags(&h->net.st, cudaStreamNonBlocking));
    cq::mlp_init(h->net, in_dim, width, out_dim, seed, h->net.st);
  });
  if (rc != COQUI_B200_OK) {
    coqui_b200_mlp_destroy(h);
    return rc;
  }
  *out = h;
  return COQUI_B200_OK;
}

void coqui_b200_mlp_destroy(coqui_b200_mlp* h) {
  if (!h) return;
  cudaSetDevice(h->net.dev);
  if (h->net.st) cudaStreamSynchronize(h->net.st);
  cudaStream_t st = h->net.st;
  delete h;  // device buffers are freed by their destructors
  if (st) cudaStreamDestroy(st);
}

const char* coqui_b200_mlp_last_error(const coqui_b200_mlp* h) { return h ? h->err.c_str() : ""; }

int64_t coqui_b200_mlp_num_params(const coqui_b200_mlp* h) { return h ? h->net.nparam : 0; }

int coqui_b200_mlp_set_params(coqui_b200_mlp* h, const float* params) {
  return mlp_guarded(h, [&] {
    CQ_REQUIRE(params, COQUI_B200_EINVAL, "null parameters");
    cq::mlp_set_params(h->net, params, h->net.st);
  });
}

int coqui_b200_mlp_get_params(coqui_b200_mlp* h, float* params) {
  return mlp_guarded(h, [&] {
    CQ_REQUIRE(params, COQUI_B200_EINVAL, "null parameters");
    CQ_CHECK_CUDA(cudaMemcpyAsync(params, h->net.w.p, h->net.nparam * sizeof(float),
                                  cudaMemcpyDeviceToHost, h->net.st));
  });
}

int coqui_b200_mlp_forward(coqui_b200_mlp* h, const float* X, int64_t B, float* Y) {
  return mlp_guarded(h, [&] {
    CQ_REQUIRE(X && Y && B >= 1, COQUI_B200_EINVAL, "bad arguments");
    cq::Mlp& n = h->net;
    cq::DevBuf<float> x, y;
    x.ensure(B * n.din);
    y.ensure(B * n.dout);
    CQ_CHECK_CUDA(cudaMemcpyAsync(x.p, X, B * n.din * sizeof(float), cudaMemcpyHostToDevice, n.st));
    cq::mlp_forward(n, x.p, B, y.p, n.st);
    CQ_CHECK_CUDA(cudaMemcpyAsync(Y, y.p, B * n.dout * sizeof(float), cudaMemcpyDeviceToHost, n.st));
    CQ_CHECK_CUDA(cudaStreamSynchronize(n.st));
  });
}

int coqui_b200_mlp_gradient(coqui_b200_mlp* h, const float* X, const float* T, int64_t B,
                            float* loss, float* grad) {
  return mlp_guarded(h, [&] {
    CQ_REQUIRE(X && T && B >= 1 && loss && grad, COQUI_B200_EINVAL, "bad arguments");
    cq::Mlp& n = h->net;
    cq::DevBuf<float> x, t;
    x.ensure(B * n.din);
    t.ensure(B * n.dout);
    CQ_CHECK_CUDA(cudaMemcpyAsync(x.p, X, B * n.din * sizeof(float), cudaMemcpyHostToDevice, n.st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(t.p, T, B * n.dout * sizeof(float), cudaMemcpyHostToDevice, n.st));
    *loss = cq::mlp_backward(n, x.p, t.p, B, n.st);
    CQ_CHECK_CUDA(cudaMemcpyAsync(grad, n.g.p, n.nparam * sizeof(float), cudaMemcpyDeviceToHost, n.st));
    CQ_CHECK_CUDA(cudaStreamSynchronize(n.st));
  });
}

int coqui_b200_mlp_extrapolate(coqui_b200_mlp* h, const double* hist, int64_t n, double max_jump,
                               double* delta) {
  return mlp_guarded(h, [&] {
    CQ_REQUIRE(hist && delta && n >= 1 && max_jump > 0, COQUI_B200_EINVAL, "bad arguments");
    cq::Mlp& net = h->net;
    cq::DevBuf<double2> dh, dd;
    dh.ensure(4 * n);
    dd.ensure(n);
    CQ_CHECK_CUDA(cudaMemcpyAsync(dh.p, hist, 4 * n * sizeof(double2), cudaMemcpyHostToDevice, net.st));
    cq::mlp_extrapolate(net, dh.p, n, max_jump, dd.p, net.st);
    CQ_CHECK_CUDA(cudaMemcpyAsync(delta, dd.p, n * sizeof(double2), cudaMemcpyDeviceToHost, net.st));
    CQ_CHECK_CUDA(cudaStreamSynchronize(net.st));
  });
}

int coqui_b200_mlp_train(coqui_b200_mlp* h, const float* X, const float* T, int64_t n_samples,
                         int64_t batch, int64_t epochs, double lr, uint64_t seed,
                         float* loss_history) {
  return mlp_guarded(h, [&] {
    CQ_REQUIRE(X && T && n_samples >= 1 && batch >= 1 && epochs >= 1, COQUI_B200_EINVAL,
               "bad arguments");
    cq::Mlp& n = h->net;
    n.xall.ensure(n_samples * n.din);
    n.tall.ensure(n_samples * n.dout);
    CQ_CHECK_CUDA(cudaMemcpyAsync(n.xall.p, X, n_samples * n.din * sizeof(float),
                                  cudaMemcpyHostToDevice, n.st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(n.tall.p, T, n_samples * n.dout * sizeof(float),
                                  cudaMemcpyHostToDevice, n.st));
    const int64_t B = std::min(batch, n_samples);
    n.idx.ensure(n_samples);
    cq::DevBuf<float> xb, tb;
    xb.ensure(B * n.din);
    tb.ensure(B * n.dout);
    std::vector<int64_t> perm(n_samples);
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937_64 rng(seed);
    for (int64_t ep = 0; ep < epochs; ++ep) {
      std::shuffle(perm.begin(), perm.end(), rng);
      CQ_CHECK_CUDA(cudaMemcpyAsync(n.idx.p, perm.data(), n_samples * sizeof(int64_t),
                                    cudaMemcpyHostToDevice, n.st));
      double sum = 0;
      int64_t nb = 0;
      for (int64_t b0 = 0; b0 + B <= n_samples; b0 += B) {
        cq::k_gather_rows<<<cq::grid_for(B * n.din, 256), 256, 0, n.st>>>(n.xall.p, n.idx.p + b0,
                                                                           xb.p, B, n.din);
        cq::k_gather_rows<<<cq::grid_for(B * n.dout, 256), 256, 0, n.st>>>(n.tall.p, n.idx.p + b0,
                                                                            tb.p, B, n.dout);
        cq::count_launch(2);
        sum += cq::mlp_backward(n, xb.p, tb.p, B, n.st);
        cq::mlp_adam_step(n, (float)lr, n.st);
        ++nb;
      }
      if (loss_history) loss_history[ep] = (float)(sum / std::max<int64_t>(nb, 1));
    }
  });
}

}  // extern "C"
