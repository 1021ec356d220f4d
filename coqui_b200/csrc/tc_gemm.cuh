// Batched complex GEMMs of the mixed-precision path (projections and Dyson products).
#pragma once

#include "common.cuh"

namespace cq {

// THC collocation X (nk, Np, nb) prepared for the projection GEMMs.
struct TcOperand {
  const double2* X = nullptr;
  int64_t nk = 0, Np = 0, nb = 0;
  DevBuf<unsigned char> packed;  // complex64 X (nk, Np, nb) then X^T (nk, nb, Np)
  DevBuf<unsigned char> tmp, tmp2;  // per-call intermediates
  void release() {
    packed.release();
    tmp.release();
    tmp2.release();
  }
};

void tc_pack_X(TcOperand& op, const double2* X, int64_t nk, int64_t Np, int64_t nb,
               cudaStream_t s);

// out[b] = X^k G^b X^k^H  (Np x Np, complex64) for nbatch problems b = (tau, k), k = b % nk;
// G (nbatch, nb, nb) complex128.
void tc_project_p2a(TcOperand& op, const double2* Gk, float2* out, int64_t nk, int64_t Np,
                    int64_t nb, int64_t nbatch, cudaStream_t s);

// out[b] = X^k^H S^b X^k  (nb x nb, complex128) for nbatch problems, k = b % nk; S (nbatch,
// Np, Np) complex64.
void tc_project_a2p(TcOperand& op, const float2* Sk, double2* out, int64_t nk, int64_t Np,
                    int64_t nb, int64_t nbatch, cudaStream_t s);

// Pre-split operand format: one float4 (hi.re, hi.im, lo.re, lo.im) per complex value with
// hi = rna_tf32(x), lo = rna_tf32(x - hi); built once for operands used by many GEMMs.
// in: nbatch blocks of (rows x cols) complex128; transpose writes each block transposed.
void to_split(const double2* in, float4* out, int64_t rows, int64_t cols, int64_t batch,
              bool transpose, cudaStream_t s);
// Complex64 copy of nbatch (rows x cols) complex128 blocks (transposed if asked).  The GEMM
// splits complex64 operands while staging them; the copy reads half the bytes of the
// pre-split format per K block, which is what bounds the long-K products.
void to_c64(const double2* in, float2* out, int64_t rows, int64_t cols, int64_t batch,
            bool transpose, cudaStream_t s);

// Split-TF32 tensor-core GEMM, "NT" form:
//   C[b](m, n) = sum_k opA(A[b])(m, k) * opB(Bt[b])(n, k)
// A: row-major M x K (lda), Bt: row-major N x K (ldb), each complex64 or pre-split (the
// *_split flags) and optionally conjugated; C: row-major complex64 (ldc).  Strides in
// complex elements; sA/sB/sC are the batch strides.
// Known zero structure lets a tile skip K blocks (and whole tiles):
//   a_upper: A(m, k) = 0 for k < m      a_lower: A(m, k) = 0 for k > m
//   b_lower: B(k, n) = 0 for k < n      b_upper: B(k, n) = 0 for k > n
//   lower_only: only tiles touching the lower triangle (m >= n) are written.
// a_mod / b_mod (> 0): the operand's batch index is (q0 + b) % mod (per-q operands shared
// by every frequency of a flattened (w, q) batch).
// a_ident / b_ident: the operand is used as (stored values + identity), with the identity on
// the operand's own diagonal (m == k for A, n == k for B); complex64 operands only.
struct TcStructure {
  bool a_upper = false, a_lower = false, b_lower = false, b_upper = false, lower_only = false;
  // tiles strictly below the diagonal are written as zeros without products (their entries
  // are not needed, and a later product may still read them)
  bool upper_zero = false;
  bool a_ident = false, b_ident = false;
  int64_t a_mod = 0, a_q0 = 0, b_mod = 0, b_q0 = 0;
};

void tc_cgemm_nt(const void* A, bool a_split, bool conj_a, int64_t lda, int64_t sA, const void* Bt,
                 bool b_split, bool conj_b, int64_t ldb, int64_t sB, float2* C, int64_t ldc,
                 int64_t sC, int64_t M, int64_t N, int64_t K, int64_t batch, cudaStream_t s,
                 const TcStructure& st = TcStructure{});

// One group of a grouped product: a batched "NT" product as tc_cgemm_nt describes.
struct TcGroup {
  const void* A = nullptr;
  bool a_split = false, conj_a = false;
  int64_t lda = 0, sA = 0;
  const void* Bt = nullptr;
  bool b_split = false, conj_b = false;
  int64_t ldb = 0, sB = 0;
  float2* C = nullptr;
  int64_t ldc = 0, sC = 0;
  int64_t M = 0, N = 0, K = 0, batch = 1;
  TcStructure st;
};

// All groups in one launch (same operand formats; the tile configuration follows the largest
// K and N).  table is the device copy of the group descriptors.
void tc_cgemm_grouped(const std::vector<TcGroup>& groups, DevBuf<unsigned char>& table,
                      cudaStream_t s);

// Tile-configuration autotuner of tc_cgemm_nt (default on; COQUI_B200_AUTOTUNE=0 or
// tc_set_autotune(0) selects the built-in heuristic) and the number of tuned shape classes.
void tc_set_autotune(int on);
int64_t tc_tuned_shapes();
// Pins the tile configuration (-1: autotuner / heuristic); false for an unknown index.
bool tc_set_forced_cfg(int cfg);
int tc_num_cfgs();

// Returns (and clears) the device flag set when a bounded wait inside a tensor-core kernel
// gave up (nonzero = a kernel timed out).
int tc_take_error();
// Whether a primary -> auxiliary projection since the last call saw NaN or Inf in G (read and
// cleared).
int tc_take_nonfinite();
// Time limit of the tensor-core kernels' bounded waits on the current device (ns; <= 0: the
// default 2 s).
void tc_set_wait_ns(int64_t ns);

}  // namespace cq
