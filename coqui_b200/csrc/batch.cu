// Uneven batch of independent Gamma-only molecules (one k-point each, different orbital and
// interpolating-point counts): one GW iteration for all of them with fused launches.
//
// Per molecule m the path is the one of the single-system context with nk = 1 (no k <-> R
// transform): G_PQ = X G X^H (thc_solver_comm.hpp:363-429), Pi = -2 G_PQ(t) o conj(G_PQ(beta-t))
// (rpa_pi.icc:156-162), tau -> iW (IAFT.icc:49-73), Dyson in Hermitian form, iW -> tau,
// Sigma_PQ = -G_PQ o W (thc_gw.icc:161-167), Sigma_ab = X^H Sigma X (thc_solver_comm.hpp:516-569).
// Fusion across molecules:
//   * every [tau][column] array concatenates the molecules' Np_m^2 columns, so the Hadamard
//     products and the IR transforms are single launches over all molecules;
//   * the projections and the Dyson products are grouped tensor-core GEMMs (one launch, one
//     group per molecule, batched over tau or iW);
//   * the FP64 factorisations of all (m, iW) problems are one grouped launch.
#include <algorithm>
#include <string>
#include <vector>

#include "chol.cuh"
#include "dyson.cuh"
#include "kernels.cuh"
#include "tc_gemm.cuh"

namespace cq {
namespace {

// Gt[m][t] = G[m][t]^T as complex64 for all molecules; offsets/edges from the molecule table
__global__ void k_transpose_grouped(const double2* __restrict__ G, float2* __restrict__ Gt,
                                    const int64_t* __restrict__ off, const int64_t* __restrict__ nb,
                                    int nmol, int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = nmol - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (off[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    const int64_t n = nb[lo], loc = i - off[lo], mat = loc / (n * n), e = loc % (n * n);
    const double2 v = G[i];
    Gt[off[lo] + mat * n * n + (e % n) * n + e / n] = make_float2((float)v.x, (float)v.y);
  }
}

struct HermProblem {
  const float2* DH;
  const float2* F;
  float2* E;
  int64_t n;
};

// E = DH + DH^H + F (F lower triangle only) for problems of different sizes: one CTA per lower
// pair of 32 x 32 tiles over the largest edge (problem blockIdx.y); pairs outside a problem
// exit at once
__global__ void __launch_bounds__(256) k_herm_sum_grouped(const HermProblem* __restrict__ probs) {
  const HermProblem pr = probs[blockIdx.y];
  int I, J;
  tile_pair((int)blockIdx.x, I, J);
  if ((int64_t)I * 32 >= pr.n) return;
  herm_sum_pair(pr.DH, pr.F, pr.E, pr.n, I, J);
}


}  // namespace
}  // namespace cq

using cq::DevBuf;

struct coqui_b200_batch {
  int dev = 0;
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;  // the one-CTA factorisations beside the tiled ones
  cudaEvent_t fork = nullptr, join = nullptr;
  std::string err;
  int64_t nmol = 0, nt = 0, nth = 0, nwb = 0, nwh = 0, nmax = 0;
  std::vector<int64_t> nb, Np;
  std::vector<int64_t> offPQ, offX, offG, offL, offD;  // element offsets per molecule
  int64_t cols = 0, nX = 0, nG = 0, nL = 0, nD = 0;
  std::vector<char> have_thc;
  bool have_ir = false;
  std::vector<double2> Twt_pos, Ttw_pos;
  DevBuf<double> dTwtR, dTtwR;
  DevBuf<float2> Xs, XTs, Ls, LHs;  // complex64 tensor-core operands
  DevBuf<double2> G, Sig, Ltmp, LHtmp;
  DevBuf<float2> Gt, T, UT, Sab, cache, PW;
  DevBuf<float2> T1, Mb, Zb, Zl;
  DevBuf<double2> Ab;
  DevBuf<int64_t> dofG, dnb;
  DevBuf<unsigned char> gtab, ctab, ctab2, htab;
  std::vector<int64_t> chol_perm;  // factorisation list position -> (molecule, iW) problem
  DevBuf<int> info;
  DevBuf<double> ld;
  DevBuf<double2> tr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0;
};

namespace {

using Batch = coqui_b200_batch;

template <typename F> int bguarded(Batch* b, F&& f) {
  if (!b) return COQUI_B200_EINVAL;
  try {
    CQ_CHECK_CUDA(cudaSetDevice(b->dev));
    f();
    if (b->st) CQ_CHECK_CUDA(cudaStreamSynchronize(b->st));
    if (cq::tc_take_error())
      throw cq::Error(COQUI_B200_ETIMEDOUT, "a tensor-core kernel gave up a bounded wait");
    b->err.clear();
    return COQUI_B200_OK;
  } catch (const cq::Error& e) {
    b->err = e.what();
    if (b->st2) (void)cudaStreamSynchronize(b->st2);
    if (b->st) (void)cudaStreamSynchronize(b->st);
    return e.code;
  } catch (const std::exception& e) {
    b->err = e.what();
    if (b->st2) (void)cudaStreamSynchronize(b->st2);
    if (b->st) (void)cudaStreamSynchronize(b->st);
    return COQUI_B200_EINVAL;
  }
}

cq::TcGroup group(const void* A, bool as, bool ca, int64_t lda, int64_t sA, const void* B, bool bs,
                  bool cb, int64_t ldb, int64_t sB, float2* C, int64_t ldc, int64_t sC, int64_t M,
                  int64_t N, int64_t K, int64_t batch, cq::TcStructure st = cq::TcStructure{}) {
  cq::TcGroup g;
  g.A = A;
  g.a_split = as;
  g.conj_a = ca;
  g.lda = lda;
  g.sA = sA;
  g.Bt = B;
  g.b_split = bs;
  g.conj_b = cb;
  g.ldb = ldb;
  g.sB = sB;
  g.C = C;
  g.ldc = ldc;
  g.sC = sC;
  g.M = M;
  g.N = N;
  g.K = K;
  g.batch = batch;
  g.st = st;
  return g;
}

// one GW iteration for all molecules; G in b->G, Sigma (complex128) into b->Sig
void batch_gw(Batch* b) {
  const cudaStream_t s = b->st;
  const int64_t nt = b->nt, nth = b->nth, nwh = b->nwh, cols = b->cols;
  // ---- G_PQ(t) = X G(t) X^H for every molecule and t (two grouped products) ----
  cq::k_transpose_grouped<<<cq::grid_for(b->nG, 256), 256, 0, s>>>(b->G.p, b->Gt.p, b->dofG.p,
                                                                   b->dnb.p, (int)b->nmol, b->nG);
  cq::count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  std::vector<cq::TcGroup> g1, g2;
  for (int64_t m = 0; m < b->nmol; ++m) {
    const int64_t nb = b->nb[m], Np = b->Np[m];
    float2* Tm = b->T.p + b->offX[m] * nt;  // (nt, Np, nb)
    g1.push_back(group(b->Xs.p + b->offX[m], false, false, nb, 0, b->Gt.p + b->offG[m], false, false,
                       nb, nb * nb, Tm, nb, Np * nb, Np, nb, nb, nt));
    g2.push_back(group(Tm, false, false, nb, Np * nb, b->Xs.p + b->offX[m], false, true, nb, 0,
                       b->cache.p + b->offPQ[m], Np, cols, Np, Np, nb, nt));
  }
  cq::tc_cgemm_grouped(g1, b->gtab, s);
  cq::tc_cgemm_grouped(g2, b->gtab, s);
  // ---- Pi(t) over all columns (nk = 1: no k <-> R transform) ----
  const cq::KGrid g0{1, 1, 1};
  for (int64_t it = 0; it < nth; ++it)
    cq::launch_pi_fused<float>(b->cache.p + it * cols, b->cache.p + (nt - 1 - it) * cols,
                               b->PW.p + it * cols, cols, g0, -2.0, s);
  cq::launch_ir_transform_real<float>(b->PW.p, cols, (int)nth, (int)nwh, b->dTwtR.p, s);
  // ---- Dyson per (m, iW): M = L^H Pi L, I - M = C C^H, W = L (D + D^H + D^H D) L^H ----
  std::vector<cq::TcGroup> p1, p2;
  for (int64_t m = 0; m < b->nmol; ++m) {
    const int64_t Np = b->Np[m], NN = Np * Np;
    cq::TcStructure s1;
    s1.a_upper = true;
    s1.upper_zero = true;  // M's lower triangle reads P1 on and above the diagonal only
    p1.push_back(group(b->LHs.p + b->offL[m], false, false, Np, 0, b->PW.p + b->offPQ[m], false, true,
                       Np, cols, b->T1.p + b->offD[m], Np, NN, Np, Np, Np, nwh, s1));
    cq::TcStructure s2;  // M = L^H (P1)^H, P1 = L^H Pi (Pi Hermitian)
    s2.a_upper = true;
    s2.lower_only = true;
    p2.push_back(group(b->LHs.p + b->offL[m], false, false, Np, 0, b->T1.p + b->offD[m], false, true,
                       Np, NN, b->Mb.p + b->offD[m], Np, NN, Np, Np, Np, nwh, s2));
  }
  cq::tc_cgemm_grouped(p1, b->gtab, s);
  cq::tc_cgemm_grouped(p2, b->gtab, s);
  std::vector<cq::CholProblem> cp;
  for (int64_t m = 0; m < b->nmol; ++m)
    for (int64_t w = 0; w < nwh; ++w) {
      const int64_t Np = b->Np[m], o = b->offD[m] + w * Np * Np;
      cp.push_back(cq::CholProblem{b->Mb.p + o, b->Ab.p + o, b->Zb.p + o, Np});
    }
  const int64_t nprob = (int64_t)cp.size();
  b->info.ensure(nprob);
  b->ld.ensure(nprob);
  b->tr.ensure(nprob);
  // FP64 factorisation with the inverse inside the kInvGroup diagonal groups only; the
  // off-group blocks of U = C^{-H} come from tensor-core doubling levels, as in the one-system
  // Dyson solve: per level bl and pair of diagonal blocks (r0: bl, r1: b1)
  //   S = U00 (-C10)^H,  U01 = S U11
  // grouped over every molecule large enough for the level.  Z = U - I, Zl = U^H - I where a
  // later level needs it, Zc = -C off the groups (in T1), S in Mb.
  std::vector<int64_t> sizes;
  for (const auto& c : cp) sizes.push_back(c.n);
  b->chol_perm.resize(nprob);
  for (int64_t i = 0; i < nprob; ++i) b->chol_perm[i] = i;
  if (cq::chol_prefer_tiled(sizes)) {
    // The largest molecules spread over many CTAs each (the tiled form, on this stream).
    // A molecule whose problems one CTA finishes within the time the tiled form needs for the
    // larger ones (n^3 x wave <= the larger molecules' sum of n^3) runs one CTA per problem on
    // the second stream at the same time, in the SMs that the tiled form's late block columns
    // (only the largest problems left) leave idle.  Same results either way.
    std::vector<int64_t> order(b->nmol);
    for (int64_t m = 0; m < b->nmol; ++m) order[m] = m;
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t x, int64_t y) { return b->Np[x] > b->Np[y]; });
    const double wave = (double)cq::chol_wave_size();
    auto cube = [&](int64_t m) { return (double)b->Np[m] * (double)b->Np[m] * (double)b->Np[m]; };
    double large = 0;
    for (int64_t m = 0; m < b->nmol; ++m) large += (double)nwh * cube(m);
    int64_t nlarge = b->nmol;
    while (nlarge > 1) {
      const int64_t m = order[nlarge - 1];
      if (cube(m) * wave > large - (double)nwh * cube(m)) break;
      large -= (double)nwh * cube(m);
      --nlarge;
    }
    std::vector<cq::CholProblem> big, small;
    int64_t pos = 0;
    for (int64_t i = 0; i < b->nmol; ++i) {
      const int64_t m = order[i];
      for (int64_t w = 0; w < nwh; ++w) {
        (i < nlarge ? big : small).push_back(cp[m * nwh + w]);
        b->chol_perm[pos++] = m * nwh + w;
      }
    }
    const int64_t nb0 = (int64_t)big.size();
    if (!small.empty()) {
      CQ_CHECK_CUDA(cudaEventRecord(b->fork, s));
      CQ_CHECK_CUDA(cudaStreamWaitEvent(b->st2, b->fork, 0));
      cq::launch_chol_inv_grouped(small, b->ctab2, b->ld.p + nb0, b->tr.p + nb0,
                                  b->info.p + nb0, b->st2, true);
      CQ_CHECK_CUDA(cudaEventRecord(b->join, b->st2));
    }
    cq::launch_chol_tiled(big, b->ctab, b->ld.p, b->tr.p, b->info.p, s);
    if (!small.empty()) CQ_CHECK_CUDA(cudaStreamWaitEvent(s, b->join, 0));
  } else {
    cq::launch_chol_inv_grouped(cp, b->ctab, b->ld.p, b->tr.p, b->info.p, s, true);
  }
  for (int64_t m = 0; m < b->nmol; ++m)
    cq::launch_chol_split(b->Ab.p + b->offD[m], b->Zb.p + b->offD[m], b->Zl.p + b->offD[m],
                          b->T1.p + b->offD[m], b->Np[m], nwh, s);
  for (int64_t bl = cq::kInvGroup; bl < b->nmax; bl *= 2) {
    struct Adj {
      int64_t m, r0, r1, b1;
    };
    std::vector<cq::TcGroup> l1, l2;
    std::vector<Adj> adj;
    for (int64_t m = 0; m < b->nmol; ++m) {
      const int64_t Np = b->Np[m], NN = Np * Np;
      if (Np <= bl) continue;
      float2* Z = b->Zb.p + b->offD[m];
      float2* Zl = b->Zl.p + b->offD[m];
      float2* Zc = b->T1.p + b->offD[m];
      float2* S = b->Mb.p + b->offD[m];
      for (int64_t r0 = 0; r0 + bl < Np; r0 += 2 * bl) {
        const int64_t r1 = r0 + bl, b1 = std::min(bl, Np - r1);
        cq::TcStructure t1;  // S = (Z + I)_00 (-C10)^H, A upper
        t1.a_upper = true;
        t1.a_ident = true;
        l1.push_back(group(Z + r0 * Np + r0, false, false, Np, NN, Zc + r1 * Np + r0, false, true,
                           Np, NN, S + r0 * Np + r1, Np, NN, bl, b1, bl, nwh, t1));
        cq::TcStructure t2;  // U01 = S U11, U11(k, n) = conj(Zl[n][k]) + delta
        t2.b_upper = true;
        t2.b_ident = true;
        l2.push_back(group(S + r0 * Np + r1, false, false, Np, NN, Zl + r1 * Np + r1, false, true,
                           Np, NN, Z + r0 * Np + r1, Np, NN, bl, b1, b1, nwh, t2));
        if (2 * bl < Np) adj.push_back(Adj{m, r0, r1, b1});
      }
    }
    cq::tc_cgemm_grouped(l1, b->gtab, s);
    cq::tc_cgemm_grouped(l2, b->gtab, s);
    for (const Adj& a : adj)
      cq::launch_block_adjoint(b->Zb.p + b->offD[a.m], b->Zl.p + b->offD[a.m], b->Np[a.m], a.r0,
                               a.r1, bl, a.b1, nwh, s);
  }
  std::vector<cq::TcGroup> f, t4, t5;
  std::vector<cq::HermProblem> hp;
  for (int64_t m = 0; m < b->nmol; ++m) {
    const int64_t Np = b->Np[m], NN = Np * Np;
    float2* Z = b->Zb.p + b->offD[m];
    float2* F = b->T1.p + b->offD[m];
    float2* E = b->Mb.p + b->offD[m];
    cq::TcStructure s3;
    s3.a_upper = true;
    s3.b_lower = true;
    s3.lower_only = true;
    f.push_back(group(Z, false, false, Np, NN, Z, false, true, Np, NN, F, Np, NN, Np, Np, Np, nwh, s3));
    for (int64_t w = 0; w < nwh; ++w)
      hp.push_back(cq::HermProblem{Z + w * NN, F + w * NN, E + w * NN, Np});
    cq::TcStructure s4;
    s4.a_lower = true;
    s4.lower_only = true;  // W is Hermitian: its lower triangle needs T only down there
    t4.push_back(group(b->Ls.p + b->offL[m], false, false, Np, 0, E, false, true, Np, NN, F, Np, NN,
                       Np, Np, Np, nwh, s4));
    cq::TcStructure s5;
    s5.b_upper = true;
    s5.lower_only = true;
    t5.push_back(group(F, false, false, Np, NN, b->Ls.p + b->offL[m], false, true, Np, 0,
                       b->PW.p + b->offPQ[m], Np, cols, Np, Np, Np, nwh, s5));
  }
  cq::tc_cgemm_grouped(f, b->gtab, s);
  CQ_REQUIRE((int64_t)hp.size() <= 65535, COQUI_B200_EINVAL, "too many Dyson problems");
  b->htab.ensure(hp.size() * sizeof(cq::HermProblem));
  CQ_CHECK_CUDA(cudaMemcpyAsync(b->htab.p, hp.data(), hp.size() * sizeof(cq::HermProblem),
                                cudaMemcpyHostToDevice, s));
  const unsigned tiles = (unsigned)((b->nmax + 31) / 32);
  cq::k_herm_sum_grouped<<<dim3(tiles * (tiles + 1) / 2, (unsigned)hp.size()), 256, 0, s>>>(
      (const cq::HermProblem*)b->htab.p);
  cq::count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  cq::tc_cgemm_grouped(t4, b->gtab, s);
  cq::tc_cgemm_grouped(t5, b->gtab, s);
  for (int64_t m = 0; m < b->nmol; ++m)  // upper triangle of W from the lower one
    cq::launch_mirror_upper(b->PW.p + b->offPQ[m], b->Np[m], nwh, s, cols);
  cq::launch_ir_transform_real<float>(b->PW.p, cols, (int)nwh, (int)nth, b->dTtwR.p, s);
  // ---- Sigma_PQ(t) = -G_PQ(t) o W(t) in place in the cache (both halves), then X^H S X ----
  for (int64_t it = 0; it < nth; ++it) {
    const bool minus = it < nt / 2;
    float2* gp = b->cache.p + it * cols;
    float2* gn = minus ? b->cache.p + (nt - 1 - it) * cols : nullptr;
    cq::launch_sigma_fused<float>(gp, gn, b->PW.p + it * cols, gp, gn, cols, g0, s);
  }
  std::vector<cq::TcGroup> a1, a2;
  for (int64_t m = 0; m < b->nmol; ++m) {
    const int64_t nb = b->nb[m], Np = b->Np[m];
    float2* U = b->UT.p + b->offX[m] * nt;  // (nt, nb, Np)
    a1.push_back(group(b->XTs.p + b->offX[m], false, false, Np, 0, b->cache.p + b->offPQ[m], false,
                       false, Np, cols, U, Np, nb * Np, nb, Np, Np, nt));
    a2.push_back(group(b->XTs.p + b->offX[m], false, true, Np, 0, U, false, false, Np, nb * Np,
                       b->Sab.p + b->offG[m], nb, nb * nb, nb, nb, Np, nt));
  }
  cq::tc_cgemm_grouped(a1, b->gtab, s);
  cq::tc_cgemm_grouped(a2, b->gtab, s);
  cq::launch_to_c128<float>(b->Sab.p, b->Sig.p, b->nG, s);
  // factorisation status
  std::vector<int> info(nprob);
  CQ_CHECK_CUDA(cudaMemcpyAsync(info.data(), b->info.p, nprob * sizeof(int), cudaMemcpyDeviceToHost, s));
  CQ_CHECK_CUDA(cudaStreamSynchronize(s));
  for (int64_t i = 0; i < nprob; ++i)
    CQ_REQUIRE(info[i] == 0, COQUI_B200_ENOTHPD,
               "I - L^H Pi L is not positive definite (problem " +
                   std::to_string(b->chol_perm[i]) + ")");
}

}  // namespace

extern "C" {

int coqui_b200_batch_create(coqui_b200_batch** out, int64_t nmol, const int64_t* nb,
                            const int64_t* Np, int64_t nt_f, int64_t nw_b, int device) {
  if (!out || nmol < 1 || !nb || !Np || nt_f < 2 || nw_b < 1) return COQUI_B200_EINVAL;
  *out = nullptr;
  for (int64_t m = 0; m < nmol; ++m)
    if (nb[m] < 1 || Np[m] < 1) return COQUI_B200_EINVAL;
  auto* b = new (std::nothrow) coqui_b200_batch();
  if (!b) return COQUI_B200_ENOMEM;
  b->dev = device;
  int rc = bguarded(b, [&] {
    // the main stream (the tiled factorisation's phases among its work) takes precedence over
    // the one-CTA factorisations that fill the SMs beside them
    int prio_least = 0, prio_greatest = 0;
    CQ_CHECK_CUDA(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
    CQ_CHECK_CUDA(cudaStreamCreateWithPriority(&b->st, cudaStreamNonBlocking, prio_greatest));
    CQ_CHECK_CUDA(cudaStreamCreateWithPriority(&b->st2, cudaStreamNonBlocking, prio_least));
    CQ_CHECK_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    CQ_CHECK_CUDA(cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming));
    CQ_CHECK_CUDA(cudaEventCreate(&b->ev0));
    CQ_CHECK_CUDA(cudaEventCreate(&b->ev1));
    b->nmol = nmol;
    b->nt = nt_f;
    b->nth = (nt_f + 1) / 2;
    b->nwb = nw_b;
    b->nwh = (nw_b + 1) / 2;
    b->nb.assign(nb, nb + nmol);
    b->Np.assign(Np, Np + nmol);
    b->have_thc.assign(nmol, 0);
    for (int64_t m = 0; m < nmol; ++m) {
      b->offPQ.push_back(b->cols);
      b->offX.push_back(b->nX);
      b->offG.push_back(b->nG);
      b->offL.push_back(b->nL);
      b->offD.push_back(b->nD);
      b->cols += Np[m] * Np[m];
      b->nX += Np[m] * nb[m];
      b->nG += nt_f * nb[m] * nb[m];
      b->nL += Np[m] * Np[m];
      b->nD += b->nwh * Np[m] * Np[m];
      b->nmax = std::max(b->nmax, Np[m]);
    }
    const int64_t nrow = std::max(b->nth, b->nwh);
    b->Xs.ensure(b->nX);
    b->XTs.ensure(b->nX);
    b->Ls.ensure(b->nL);
    b->LHs.ensure(b->nL);
    b->G.ensure(b->nG);
    b->Sig.ensure(b->nG);
    b->Gt.ensure(b->nG);
    b->Sab.ensure(b->nG);
    b->T.ensure(b->nX * nt_f);
    b->UT.ensure(b->nX * nt_f);
    b->cache.ensure(nt_f * b->cols);
    b->PW.ensure(nrow * b->cols);
    b->T1.ensure(b->nD);
    b->Mb.ensure(b->nD);
    b->Zb.ensure(b->nD);
    b->Zl.ensure(b->nD);
    b->Ab.ensure(b->nD);
    std::vector<int64_t> offs(b->offG);
    b->dofG.ensure(nmol);
    b->dnb.ensure(nmol);
    CQ_CHECK_CUDA(cudaMemcpyAsync(b->dofG.p, offs.data(), nmol * sizeof(int64_t),
                                  cudaMemcpyHostToDevice, b->st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(b->dnb.p, b->nb.data(), nmol * sizeof(int64_t),
                                  cudaMemcpyHostToDevice, b->st));
  });
  if (rc != COQUI_B200_OK) {
    coqui_b200_batch_destroy(b);
    return rc;
  }
  *out = b;
  return COQUI_B200_OK;
}

void coqui_b200_batch_destroy(coqui_b200_batch* b) {
  if (!b) return;
  cudaSetDevice(b->dev);
  if (b->st2) cudaStreamSynchronize(b->st2);
  if (b->st) cudaStreamSynchronize(b->st);
  cudaStream_t st = b->st, st2 = b->st2;
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->join) cudaEventDestroy(b->join);
  delete b;
  if (st) cudaStreamDestroy(st);
  if (st2) cudaStreamDestroy(st2);
}

double coqui_b200_batch_last_ms(const coqui_b200_batch* b) { return b ? b->last_ms : 0.0; }

const char* coqui_b200_batch_last_error(const coqui_b200_batch* b) {
  return b ? b->err.c_str() : "";
}

int coqui_b200_batch_set_ir(coqui_b200_batch* b, const double* Twt_bb, const double* Ttw_bb,
                            const double* tau_mesh_x) {
  return bguarded(b, [&] {
    CQ_REQUIRE(Twt_bb && Ttw_bb && tau_mesh_x, COQUI_B200_EINVAL, "null IR table");
    const int64_t nt = b->nt;
    for (int64_t it = 0; it < nt; ++it)
      CQ_REQUIRE(std::abs(std::abs(tau_mesh_x[it]) - std::abs(tau_mesh_x[nt - it - 1])) <= 1e-6,
                 COQUI_B200_EPHSYM, "IAFT grid is not compatible with particle-hole symmetry");
    cq::ph_symmetric_matrices(Twt_bb, Ttw_bb, nt, b->nwb, b->Twt_pos, b->Ttw_pos);
    double re = 0, im = 0;
    for (const auto* v : {&b->Twt_pos, &b->Ttw_pos})
      for (const double2& z : *v) {
        re = std::max(re, std::abs(z.x));
        im = std::max(im, std::abs(z.y));
      }
    CQ_REQUIRE(im <= 1e-12 * re, COQUI_B200_EUNSUPPORTED,
               "the batched path needs real particle-hole symmetric IR matrices");
    std::vector<double> a(b->Twt_pos.size()), c(b->Ttw_pos.size());
    for (size_t i = 0; i < a.size(); ++i) a[i] = b->Twt_pos[i].x;
    for (size_t i = 0; i < c.size(); ++i) c[i] = b->Ttw_pos[i].x;
    b->dTwtR.ensure(a.size());
    b->dTtwR.ensure(c.size());
    CQ_CHECK_CUDA(cudaMemcpyAsync(b->dTwtR.p, a.data(), a.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, b->st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(b->dTtwR.p, c.data(), c.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, b->st));
    CQ_CHECK_CUDA(cudaStreamSynchronize(b->st));
    b->have_ir = true;
  });
}

int coqui_b200_batch_set_thc(coqui_b200_batch* b, int64_t m, const double* X_Pa, const double* V_PQ) {
  return bguarded(b, [&] {
    CQ_REQUIRE(m >= 0 && m < b->nmol && X_Pa && V_PQ, COQUI_B200_EINVAL, "bad arguments");
    const int64_t Np = b->Np[m], nb = b->nb[m];
    DevBuf<double2> X, L, LH;
    X.ensure(Np * nb);
    L.ensure(Np * Np);
    LH.ensure(Np * Np);
    CQ_CHECK_CUDA(cudaMemcpyAsync(X.p, X_Pa, Np * nb * sizeof(double2), cudaMemcpyHostToDevice, b->st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(L.p, V_PQ, Np * Np * sizeof(double2), cudaMemcpyHostToDevice, b->st));
    const int info = cq::cholesky_lower_batched(L.p, Np, 1, b->st);
    CQ_REQUIRE(info == 0, COQUI_B200_ENOTHPD, "Coulomb matrix V is not positive definite");
    cq::launch_zero_upper_and_adjoint(L.p, LH.p, Np, 1, b->st);
    cq::to_c64(X.p, b->Xs.p + b->offX[m], Np, nb, 1, false, b->st);
    cq::to_c64(X.p, b->XTs.p + b->offX[m], Np, nb, 1, true, b->st);
    cq::to_c64(L.p, b->Ls.p + b->offL[m], Np, Np, 1, false, b->st);
    cq::to_c64(LH.p, b->LHs.p + b->offL[m], Np, Np, 1, false, b->st);
    CQ_CHECK_CUDA(cudaStreamSynchronize(b->st));
    b->have_thc[m] = 1;
  });
}

int coqui_b200_batch_gw_iteration(coqui_b200_batch* b, const double* const* G_list,
                                  double* const* Sigma_list) {
  return bguarded(b, [&] {
    CQ_REQUIRE(b->have_ir, COQUI_B200_EINVAL, "batch_set_ir not called");
    for (int64_t m = 0; m < b->nmol; ++m)
      CQ_REQUIRE(b->have_thc[m], COQUI_B200_EINVAL, "batch_set_thc not called for every molecule");
    CQ_REQUIRE(G_list, COQUI_B200_EINVAL, "null G list");
    for (int64_t m = 0; m < b->nmol; ++m) {
      CQ_REQUIRE(G_list[m], COQUI_B200_EINVAL, "null G");
      CQ_CHECK_CUDA(cudaMemcpyAsync(b->G.p + b->offG[m], G_list[m],
                                    b->nt * b->nb[m] * b->nb[m] * sizeof(double2),
                                    cudaMemcpyHostToDevice, b->st));
    }
    CQ_CHECK_CUDA(cudaEventRecord(b->ev0, b->st));
    batch_gw(b);
    CQ_CHECK_CUDA(cudaEventRecord(b->ev1, b->st));
    CQ_CHECK_CUDA(cudaEventSynchronize(b->ev1));
    float ms = 0;
    CQ_CHECK_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->last_ms = ms;
    if (Sigma_list)
      for (int64_t m = 0; m < b->nmol; ++m)
        if (Sigma_list[m])
          CQ_CHECK_CUDA(cudaMemcpyAsync(Sigma_list[m], b->Sig.p + b->offG[m],
                                        b->nt * b->nb[m] * b->nb[m] * sizeof(double2),
                                        cudaMemcpyDeviceToHost, b->st));
    // page-locked destinations: the copies above return at once; the call returns after they
    // landed, as every entry point of the library does
    CQ_CHECK_CUDA(cudaStreamSynchronize(b->st));
  });
}

}  // extern "C"
