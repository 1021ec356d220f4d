// Launchers of the SIMT kernels of the THC-RPA/GW path (kernels.cu).
#pragma once

#include "common.cuh"

namespace cq {

// k-mesh of a Gamma-centred Monkhorst-Pack grid; k = (i0 * n1 + i1) * n2 + i2.
struct KGrid {
  int n0, n1, n2;
  int nk() const { return n0 * n1 * n2; }
};

void upload_twiddles();

// Pi(tau) columns: Pi[q, c] = sp * IDFT_R->q( DFT_k->R(Gp)[R, c] * conj(DFT_k->R(Gn)[R, c]) )
// with the reference's normalisation (f_Rk = e^{-ikR}/nk, f_qR = e^{+iqR}).
// Arrays are (nk, ncol) row-major in storage precision R.
template <typename R>
void launch_pi_fused(const cplx_t<R>* Gp, const cplx_t<R>* Gn, cplx_t<R>* Pi, int64_t ncol,
                     KGrid g, double sp, cudaStream_t s);

// Sigma(tau) and Sigma(beta - tau) columns from G(tau), G(beta - tau) and W_R(tau):
// S = IDFT_R->k( -DFT_k->R(G) * W_R ).  Sm/Gm may be null (skipped).
template <typename R>
void launch_sigma_fused(const cplx_t<R>* Gp, const cplx_t<R>* Gm, const cplx_t<R>* WR,
                        cplx_t<R>* Sp, cplx_t<R>* Sm, int64_t ncol, KGrid g, cudaStream_t s);

// In-place 3D DFT over the leading k index of nbatch blocks of (nk, ncol):
// sign = -1 with scale 1/nk is f_Rk; sign = +1 with scale 1 is f_kR.
template <typename R>
void launch_dft_plain(cplx_t<R>* buf, int64_t ncol, KGrid g, int sign, double scale,
                      int64_t nbatch, int64_t batch_stride, cudaStream_t s);

// In-place transform along the leading index: buf[n, e] = sum_t M[n, t] buf[t, e],
// t < n_in, n < n_out; buf has room for max(n_in, n_out) leading rows; M is complex128
// (n_out, n_in) on the device.
template <typename R>
void launch_ir_transform(cplx_t<R>* buf, int64_t ncol, int n_in, int n_out, const double2* M,
                         cudaStream_t s);

// Same with a real matrix M (n_out, n_in) (FP64).
template <typename R>
void launch_ir_transform_real(cplx_t<R>* buf, int64_t ncol, int n_in, int n_out, const double* M,
                              cudaStream_t s);

// complex128 -> storage precision (and back) element-wise conversions.
template <typename R>
void launch_from_c128(const double2* in, cplx_t<R>* out, int64_t n, cudaStream_t s);
template <typename R>
void launch_to_c128(const cplx_t<R>* in, double2* out, int64_t n, cudaStream_t s);

// A[p] = I - M[p] (complex128 out) for nprob Np x Np problems.
template <typename R>
void launch_eye_minus(const cplx_t<R>* M, double2* A, int64_t Np, int64_t nprob, cudaStream_t s);

// For each problem p: logdet[p] = 2 sum_i ln Re C_ii (C lower Cholesky factor, complex128),
// trace[p] = sum_i M_ii (complex).
template <typename R>
void launch_logdet_trace(const double2* C, const cplx_t<R>* M, double* logdet, double2* trace,
                         int64_t Np, int64_t nprob, cudaStream_t s);

// eps(t, q) = fac[q] * sum_PQ chi[q, P] W[t, q, P, Q] conj(chi[q, Q]); W in storage precision.
template <typename R>
void launch_eps_head(const cplx_t<R>* W, const double2* chi, const double* fac, double2* eps,
                     int64_t nt, int64_t nq, int64_t Np, cudaStream_t s);

// W (nt, nq, ncol) storage -> out (nq, nt, ncol) complex128 for q in [q0, q0 + nqc).
template <typename R>
void launch_tq_to_qt_c128(const cplx_t<R>* W, double2* out, int64_t nt, int64_t nq,
                          int64_t ncol, int64_t q0, int64_t nqc, cudaStream_t s);
// in (nq, nt, ncol) complex128 -> W (nt, nq, ncol) storage.
template <typename R>
void launch_qt_to_tq(const double2* in, cplx_t<R>* W, int64_t nt, int64_t nq, int64_t ncol,
                     cudaStream_t s);

// Batched complex GEMM on CUDA cores with general strides (used where no tensor-core
// kernel applies): C[b] = alpha * opA(A[b]) * opB(B[b]) + beta * C[b] where
// opA(A)(m, k) = A[m * sam + k * sak] (conjugated if conj_a), same for B with (k, n).
struct GemmDesc {
  int64_t M, N, K;
  int64_t sam, sak, sbk, sbn, scm, scn;
  int64_t batch, bsa, bsb, bsc;
  bool conj_a, conj_b;
  double2 alpha, beta;
};
template <typename TA, typename TB, typename TC, typename Acc>
void launch_gemm_simt(const GemmDesc& d, const TA* A, const TB* B, TC* C, cudaStream_t s);

// Particle-hole symmetric IR matrices (IAFT.icc:61-70 tau -> w, :116-125 w -> tau; nt_b() is
// nt_f, IAFT.hpp:167-169) from the bosonic tables Twt_bb (nwb, nt), Ttw_bb (nt, nwb) given as
// (re, im) pairs: Twt_pos (nwh, nth), Ttw_pos (nth, nwh).
void ph_symmetric_matrices(const double* Twt_bb, const double* Ttw_bb, int64_t nt, int64_t nwb,
                           std::vector<double2>& Twt_pos, std::vector<double2>& Ttw_pos);

// *flag = 1 if any of the n complex values holds NaN or Inf (flag left as it is otherwise).
void launch_check_finite(const double2* p, int64_t n, int* flag, cudaStream_t s);

}  // namespace cq
