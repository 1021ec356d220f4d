// Shared helpers of the THC-RPA/GW device library: complex types, status propagation,
// launch accounting and the small fixed-size DFT twiddle table.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <cuComplex.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/coqui_b200.h"

namespace cq {

// Status carried by exceptions inside the library; converted to return codes at the ABI.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CQ_CHECK_CUDA(expr)                                                              \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess)                                                               \
      throw ::cq::Error(_e == cudaErrorMemoryAllocation ? COQUI_B200_ENOMEM              \
                                                        : COQUI_B200_ECUDA,              \
                        std::string(#expr) + ": " + cudaGetErrorString(_e));             \
  } while (0)

#define CQ_REQUIRE(cond, code, msg)         \
  do {                                      \
    if (!(cond)) throw ::cq::Error(code, msg); \
  } while (0)

// Device complex value type selected by the storage precision.
template <typename R> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };
template <typename R> using cplx_t = typename Cplx<R>::type;

template <typename C> __host__ __device__ __forceinline__ C mk(double re, double im) {
  C c;
  c.x = re;
  c.y = im;
  return c;
}
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) {
  C c; c.x = a.x + b.x; c.y = a.y + b.y; return c;
}
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) {
  C c; c.x = a.x - b.x; c.y = a.y - b.y; return c;
}
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  C c; c.x = a.x * b.x - a.y * b.y; c.y = a.x * b.y + a.y * b.x; return c;
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
  C c; c.x = a.x * b.x + a.y * b.y; c.y = a.y * b.x - a.x * b.y; return c;
}
template <typename C, typename R> __host__ __device__ __forceinline__ C cscale(C a, R s) {
  C c; c.x = a.x * s; c.y = a.y * s; return c;
}

// Grid-size helper: enough blocks to cover n items, capped to keep launches modest.
inline unsigned grid_for(int64_t n, int block, int64_t cap = 148 * 64) {
  int64_t g = (n + block - 1) / block;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

// Grow-only device buffer owned by a context.
template <typename T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void ensure(size_t count) {
    if (count <= n) return;
    release();
    cudaError_t e = cudaMalloc((void**)&p, (count ? count : 1) * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();  // the failed allocation is not a sticky error: clear it
      throw Error(COQUI_B200_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    n = count;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Optional per-kernel CUDA-event timing on the launching stream (off by default).
struct Prof {
  bool on = false;
  cudaStream_t st = nullptr;
  std::vector<std::tuple<std::string, cudaEvent_t, cudaEvent_t, int64_t>> pending;
  // name -> (ms, launch groups, work units: the problems a group processed, where it counts them)
  std::map<std::string, std::tuple<double, int64_t, int64_t>> acc;
  struct Scope {
    Prof* p = nullptr;
    std::string name;
    cudaEvent_t a = nullptr;
    int64_t units = 0;
    Scope(Prof* pr, const char* n, int64_t u = 0) : p(pr && pr->on ? pr : nullptr), name(n), units(u) {
      if (p) {
        nvtxRangePushA(n);  // profilers can select the group's kernels by this range
        cudaEventCreate(&a);
        cudaEventRecord(a, p->st);
      }
    }
    Scope(const Scope&) = delete;
    ~Scope() {
      if (!p) return;
      nvtxRangePop();
      cudaEvent_t b;
      cudaEventCreate(&b);
      cudaEventRecord(b, p->st);
      p->pending.emplace_back(name, a, b, units);
    }
  };
  // call after the stream has been synchronised
  void resolve() {
    for (auto& t : pending) {
      float ms = 0;
      cudaEventElapsedTime(&ms, std::get<1>(t), std::get<2>(t));
      auto& e = acc[std::get<0>(t)];
      std::get<0>(e) += ms;
      std::get<1>(e) += 1;
      std::get<2>(e) += std::get<3>(t);
      cudaEventDestroy(std::get<1>(t));
      cudaEventDestroy(std::get<2>(t));
    }
    pending.clear();
  }
};

// Kernels launched by this library (all contexts); read by coqui_b200_kernel_launches.
int64_t launches_total();
void count_launch(int64_t n = 1);

}  // namespace cq
