// Allocation-free variant of the tensor-core primary -> auxiliary projection
//   O^k_PQ = X^k_Pa G^k_ab conj(X^k_Qb).
//
// Who needs it: code that owns its device buffers but may not allocate device memory --
// a host application whose memory is handed out by its own pool or arena, a caller that
// holds a fixed device-memory budget, or code running where cudaMalloc/cudaFree would
// synchronise the device at the wrong moment.  Such a caller passes device pointers for the
// inputs and the output; every intermediate of the projection (the pre-split X, X G and
// G^T) lives in one statically sized device array that this file declares.
//
// Limits and sharing:
//   * the scratch array is kNoAllocScratchBytes (32 MiB); problems that need more are
//     rejected with COQUI_B200_EINVAL and a message naming the required size;
//   * every device that loads the library holds the array until the process exits;
//   * all calls share the array and it keeps the last call's contents; each call overwrites
//     every scratch byte it reads before reading it, so nothing has to be cleared, but two
//     calls whose work overlaps on the GPU (different streams, or different host threads)
//     race on the array;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (a host-side use of the array's name is not a device address);
//     make that first call before any stream capture.
#include <cstdio>
#include <mutex>

#include "kernels.cuh"
#include "tc_gemm.cuh"

namespace cq {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per device).
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

// out[k] = G[k]^T as complex64 (nb x nb blocks of complex128)
__global__ void k_noalloc_transpose(const double2* __restrict__ in, float2* __restrict__ out,
                                    int64_t nb, int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = i / (nb * nb), e = i % (nb * nb);
    const double2 x = in[i];
    out[k * nb * nb + (e % nb) * nb + e / nb] = make_float2((float)x.x, (float)x.y);
  }
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

void set_msg(char* buf, int len, const char* msg) {
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", msg);
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// a * b * c * elem bytes, or false when that exceeds `limit`.  Each factor is compared with
// the limit divided by the product so far, so no multiplication can wrap around.
bool bytes_within(size_t a, size_t b, size_t c, size_t elem, size_t limit, size_t* out) {
  size_t room = limit / elem;
  if (a > room) return false;
  room /= a;
  if (b > room) return false;
  room /= b;
  if (c > room) return false;
  *out = a * b * c * elem;
  return true;
}

}  // namespace
}  // namespace cq

extern "C" COQUI_B200_API int coqui_b200_primary_to_aux_noalloc(
    const double* X_skPa, const double* O_skab, float* O_skPQ, int64_t nk, int64_t Np,
    int64_t nb, void* stream, char* errbuf, int errlen) {
  using namespace cq;
  set_msg(errbuf, errlen, "");
  if (nk < 1 || Np < 1 || nb < 1) {
    set_msg(errbuf, errlen, "nk, Np and nb must be positive");
    return COQUI_B200_EINVAL;
  }
  // Every size is checked against the limit before it is formed (no wrap-around for huge
  // dimensions); each part is at most the limit, so their aligned sum cannot wrap either.
  size_t raw_xs = 0, raw_t = 0, raw_gt = 0;
  const size_t lim = kNoAllocScratchBytes;
  const bool fits = bytes_within(nk, Np, nb, sizeof(float4), lim, &raw_xs) &&
                    bytes_within(nk, Np, nb, sizeof(float2), lim, &raw_t) &&
                    bytes_within(nk, nb, nb, sizeof(float2), lim, &raw_gt);
  const size_t bytes_xs = align256(raw_xs), bytes_t = align256(raw_t),
               bytes_gt = align256(raw_gt);
  if (!fits || bytes_xs + bytes_t + bytes_gt > lim) {
    char m[224];
    if (fits)
      std::snprintf(m, sizeof(m),
                    "problem needs %zu bytes of scratch; the static limit is %zu bytes (32 MiB)",
                    bytes_xs + bytes_t + bytes_gt, lim);
    else
      std::snprintf(m, sizeof(m),
                    "problem (nk %lld, Np %lld, nb %lld) exceeds the static limit of %zu bytes "
                    "(32 MiB) of scratch",
                    (long long)nk, (long long)Np, (long long)nb, lim);
    set_msg(errbuf, errlen, m);
    return COQUI_B200_EINVAL;
  }
  if (!X_skPa || !O_skab || !O_skPQ || !is_device_pointer(X_skPa) ||
      !is_device_pointer(O_skab) || !is_device_pointer(O_skPQ)) {
    set_msg(errbuf, errlen, "X, G and the output must be device pointers");
    return COQUI_B200_EINVAL;
  }
  try {
    void* base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess) {
      set_msg(errbuf, errlen, cudaGetErrorString(e));
      return COQUI_B200_ECUDA;
    }
    unsigned char* sp = static_cast<unsigned char*>(base);
    float4* Xs = reinterpret_cast<float4*>(sp);
    float2* T = reinterpret_cast<float2*>(sp + bytes_xs);
    float2* Gt = reinterpret_cast<float2*>(sp + bytes_xs + bytes_t);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const double2* X = reinterpret_cast<const double2*>(X_skPa);
    const double2* G = reinterpret_cast<const double2*>(O_skab);
    float2* out = reinterpret_cast<float2*>(O_skPQ);

    to_split(X, Xs, Np, nb, nk, false, s);
    const int64_t tg = nk * nb * nb;
    k_noalloc_transpose<<<grid_for(tg, 256), 256, 0, s>>>(G, Gt, nb, tg);
    count_launch();
    CQ_CHECK_CUDA(cudaGetLastError());
    // T = X G (Np x nb), then O = T X^H (Np x Np)
    tc_cgemm_nt(Xs, true, false, nb, Np * nb, Gt, false, false, nb, nb * nb, T, nb, Np * nb, Np,
                nb, nb, nk, s);
    tc_cgemm_nt(T, false, false, nb, Np * nb, Xs, true, true, nb, Np * nb, out, Np, Np * Np, Np,
                Np, nb, nk, s);
    CQ_CHECK_CUDA(cudaStreamSynchronize(s));
    if (tc_take_error()) {
      set_msg(errbuf, errlen, "a tensor-core kernel gave up a bounded wait");
      return COQUI_B200_ETIMEDOUT;
    }
  } catch (const Error& err) {
    set_msg(errbuf, errlen, err.what());
    return err.code;
  }
  return COQUI_B200_OK;
}
