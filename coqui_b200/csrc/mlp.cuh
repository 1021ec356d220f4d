// Small multilayer perceptron (in -> width -> width -> out, tanh activations) with BF16
// weights and FP32 accumulation: hand-written forward, backward and Adam kernels.  It proposes
// the next self-energy update of the self-consistent GW loop from the last iterates.
#pragma once

#include <cuda_bf16.h>

#include <vector>

#include "common.cuh"

namespace cq {

struct Mlp {
  int64_t din = 0, width = 0, dout = 0;
  int64_t nparam = 0;
  int dev = 0;
  cudaStream_t st = nullptr;
  DevBuf<float> w;              // FP32 master parameters: W1 b1 W2 b2 W3 b3
  DevBuf<__nv_bfloat16> wb;     // BF16 copy used by the forward pass (biases too)
  DevBuf<float> g, m, v;        // gradient and Adam moments
  int64_t adam_t = 0;
  // activations of the last forward pass (batch capacity cap)
  int64_t cap = 0;
  DevBuf<float> x, h1, h2, y, t, dy, dh2, dh1, part;
  DevBuf<int64_t> idx;
  DevBuf<float> xall, tall;     // training set (device)
  int64_t nall = 0;

  // parameter offsets (elements)
  int64_t oW1() const { return 0; }
  int64_t ob1() const { return width * din; }
  int64_t oW2() const { return ob1() + width; }
  int64_t ob2() const { return oW2() + width * width; }
  int64_t oW3() const { return ob2() + width; }
  int64_t ob3() const { return oW3() + dout * width; }
};

void mlp_init(Mlp& n, int64_t din, int64_t width, int64_t dout, uint64_t seed, cudaStream_t s);
// parameters from FP32 host values (rounded to BF16 for the forward pass)
void mlp_set_params(Mlp& n, const float* host, cudaStream_t s);
// y (B, dout) = MLP(x) for device x (B, din); activations kept for a backward pass
void mlp_forward(Mlp& n, const float* x, int64_t B, float* y, cudaStream_t s);
// loss = mean (y - t)^2 over B x dout and the gradient of every parameter into n.g
float mlp_backward(Mlp& n, const float* x, const float* t, int64_t B, cudaStream_t s);
void mlp_adam_step(Mlp& n, float lr, cudaStream_t s);

// Learned extrapolation of nel sequences from their last four iterates hist (4, nel)
// complex128 (oldest first): with d1 = s3 - s2, d2 = s2 - s1, d3 = s1 - s0 the network maps
// (d1/d2, d2/d3) to (s_inf - s3)/d1; delta = d1 * output, |delta| <= max_jump |d1|, and 0 where
// the differences vanish.
void mlp_extrapolate(Mlp& n, const double2* hist, int64_t nel, double max_jump, double2* delta,
                     cudaStream_t s);

}  // namespace cq

struct coqui_b200_mlp;
cq::Mlp& mlp_net(coqui_b200_mlp* h);
