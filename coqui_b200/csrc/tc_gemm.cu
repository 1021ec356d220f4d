// Mixed-precision batched complex GEMMs (projections, Dyson products).
#include "kernels.cuh"
#include "tc_gemm.cuh"

namespace cq {

namespace {

// opA(A)(m, k) for row-major storage: N -> A[m][k] (lda = K), C -> conj(A[k][m]) (lda = M)
void set_a(GemmDesc& d, TcOp op, int64_t M, int64_t K) {
  if (op == TcOp::N) {
    d.sam = K;
    d.sak = 1;
    d.conj_a = false;
  } else {
    d.sam = 1;
    d.sak = M;
    d.conj_a = true;
  }
}
void set_b(GemmDesc& d, TcOp op, int64_t K, int64_t N) {
  if (op == TcOp::N) {
    d.sbk = N;
    d.sbn = 1;
    d.conj_b = false;
  } else {
    d.sbk = 1;
    d.sbn = K;
    d.conj_b = true;
  }
}

}  // namespace

void tc_pack_X(TcOperand& op, const double2* X, int64_t nk, int64_t Np, int64_t nb,
               cudaStream_t) {
  op.X = X;
  op.nk = nk;
  op.Np = Np;
  op.nb = nb;
}

void tc_project_p2a(TcOperand& op, const double2* Gk, float2* out, int64_t nk, int64_t Np,
                    int64_t nb, cudaStream_t s) {
  op.tmp.ensure((size_t)nk * Np * nb * sizeof(float2));
  float2* T = (float2*)op.tmp.p;
  GemmDesc d{};
  // T = X G  (Np x nb, K = nb)
  d.M = Np; d.N = nb; d.K = nb;
  set_a(d, TcOp::N, Np, nb);
  set_b(d, TcOp::N, nb, nb);
  d.scm = nb; d.scn = 1;
  d.batch = nk; d.bsa = Np * nb; d.bsb = nb * nb; d.bsc = Np * nb;
  d.alpha = make_double2(1, 0); d.beta = make_double2(0, 0);
  launch_gemm_simt<double2, double2, float2, float>(d, op.X, Gk, T, s);
  // out = T X^H  (Np x Np, K = nb)
  GemmDesc e{};
  e.M = Np; e.N = Np; e.K = nb;
  set_a(e, TcOp::N, Np, nb);
  set_b(e, TcOp::C, nb, Np);
  e.scm = Np; e.scn = 1;
  e.batch = nk; e.bsa = Np * nb; e.bsb = Np * nb; e.bsc = Np * Np;
  e.alpha = make_double2(1, 0); e.beta = make_double2(0, 0);
  launch_gemm_simt<float2, double2, float2, float>(e, T, op.X, out, s);
}

void tc_project_a2p(TcOperand& op, const float2* Sk, double2* out, int64_t nk, int64_t Np,
                    int64_t nb, cudaStream_t s) {
  op.tmp.ensure((size_t)nk * Np * nb * sizeof(float2));
  float2* T = (float2*)op.tmp.p;
  GemmDesc d{};
  // T = X^H S  (nb x Np, K = Np)
  d.M = nb; d.N = Np; d.K = Np;
  set_a(d, TcOp::C, nb, Np);
  set_b(d, TcOp::N, Np, Np);
  d.scm = Np; d.scn = 1;
  d.batch = nk; d.bsa = Np * nb; d.bsb = Np * Np; d.bsc = nb * Np;
  d.alpha = make_double2(1, 0); d.beta = make_double2(0, 0);
  launch_gemm_simt<double2, float2, float2, float>(d, op.X, Sk, T, s);
  // out = T X  (nb x nb, K = Np)
  GemmDesc e{};
  e.M = nb; e.N = nb; e.K = Np;
  set_a(e, TcOp::N, nb, Np);
  set_b(e, TcOp::N, Np, nb);
  e.scm = nb; e.scn = 1;
  e.batch = nk; e.bsa = nb * Np; e.bsb = Np * nb; e.bsc = nb * nb;
  e.alpha = make_double2(1, 0); e.beta = make_double2(0, 0);
  launch_gemm_simt<float2, double2, double2, double>(e, T, op.X, out, s);
}

template <typename TA, typename TB>
void tc_gemm_c(TcOp opa, const TA* A, TcOp opb, const TB* B, float2* C, int64_t M, int64_t N,
               int64_t K, int64_t batch, cudaStream_t s, bool minus_c) {
  GemmDesc d{};
  d.M = M; d.N = N; d.K = K;
  set_a(d, opa, M, K);
  set_b(d, opb, K, N);
  d.scm = N; d.scn = 1;
  d.batch = batch; d.bsa = M * K; d.bsb = K * N; d.bsc = M * N;
  d.alpha = make_double2(1, 0);
  d.beta = minus_c ? make_double2(-1, 0) : make_double2(0, 0);
  launch_gemm_simt<TA, TB, float2, float>(d, A, B, C, s);
}

template void tc_gemm_c<float2, double2>(TcOp, const float2*, TcOp, const double2*, float2*,
                                         int64_t, int64_t, int64_t, int64_t, cudaStream_t, bool);
template void tc_gemm_c<double2, float2>(TcOp, const double2*, TcOp, const float2*, float2*,
                                         int64_t, int64_t, int64_t, int64_t, cudaStream_t, bool);
template void tc_gemm_c<double2, double2>(TcOp, const double2*, TcOp, const double2*, float2*,
                                          int64_t, int64_t, int64_t, int64_t, cudaStream_t, bool);

}  // namespace cq
