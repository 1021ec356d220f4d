// Host side of the symmetry-reduced (IBZ) k-space path; part of ctx.cu (included there, after
// the pipeline helpers it uses).
//
// Reference: scr_coulomb_t::eval_Pi_rpa_kspace (src/methods/scr_coulomb/rpa_pi.icc:182-336),
// gw_t::eval_Sigma_all_kspace (src/methods/GW/thc_gw.icc:216-443) and the IBZ-weighted RPA
// energy (src/methods/GW/thc_rpa.icc:130-173), with thc_solver_comm::primary_to_aux taking the
// IBZ matrices through kp_to_ibz / kp_trev (thc_solver_comm.hpp:405-428).
//
//   G (IBZ k) --unfold (kp_to_ibz, transposed for time-reversal images)--> G (all k)
//   Pi_q for every q on the R-space route, then Pi^k(q) = transpose(Pi^R(-q)) for the IBZ q
//     (the reference's k-space sum, sum_k conj(G(k-q, t)) G(k, beta-t), is that transpose)
//   tau -> iW, Dyson with V of the IBZ q-points, iW -> tau          (nq_ibz problems per iW)
//   Sigma(k_ibz) = sum_isym D^H [X^H(ks) S_isym X(ks)] D,  ks = ks_to_k(isym, k),
//     S_isym = -1/nk sum_{q in Qs(isym)} G(ks -+ qs) * W(qs) with the reference's conjugations
//
// The polarizability takes the R-space route because the fused DFT kernels make it one pass
// over G per tau, where the reference's k-space double loop costs nq_ibz * nk element products;
// both give the same sums.  The self-energy keeps the reference's term lists: per tau slice one
// pass stages each column tile of every G(k) and W(q_ibz) in shared memory and forms the rows
// of all (isym, k_ibz) from there, so G and W cross HBM once however many terms read them.
// defined further down in ctx.cu, inside its extern "C" block (shared with the full-BZ route)
extern "C" {
namespace {
void select_head_from(Ctx* c, const std::vector<double2>& eps, int64_t nq,
                      const std::vector<double>& qnorm, const std::vector<double>& qz,
                      int64_t q_smallest);
void sigma_div_correction_on(Ctx* c, int64_t nk, const double2* X, const double2* G,
                             double2* Sig, DevBuf<double2>& Tdiv, bool& tdiv_valid);
}  // namespace
}

namespace {

void lex_coords(const Ctx* c, int64_t p, int64_t x[3]) {
  x[0] = p / ((int64_t)c->g.n1 * c->g.n2);
  x[1] = (p / c->g.n2) % c->g.n1;
  x[2] = p % c->g.n2;
}
int64_t lex_pos(const Ctx* c, const int64_t x[3]) {
  const int64_t n[3] = {c->g.n0, c->g.n1, c->g.n2};
  int64_t y[3];
  for (int i = 0; i < 3; ++i) y[i] = ((x[i] % n[i]) + n[i]) % n[i];
  return (y[0] * n[1] + y[1]) * n[2] + y[2];
}
// lexicographic position of k_a - k_b (+ s k_b for s = +1: k_a + k_b)
int64_t lex_combine(const Ctx* c, int64_t pa, int64_t pb, int s) {
  int64_t a[3], b[3], r[3];
  lex_coords(c, pa, a);
  lex_coords(c, pb, b);
  for (int i = 0; i < 3; ++i) r[i] = a[i] + s * b[i];
  return lex_pos(c, r);
}

// X at ks_to_k and the Coulomb factors at the IBZ q-points, from the current THC data
void sym_prepare_thc(Ctx* c) {
  SymState& S = *c->sym;
  if (S.thc_ready) return;
  CQ_REQUIRE(c->have_thc, COQUI_B200_EINVAL, "set_thc not called");
  const int64_t nki = S.nk_ibz, nqi = S.nq_ibz, Np = c->Np, nb = c->nb;
  const int64_t per = Np * nb, pp = Np * Np;
  S.Xs.ensure((size_t)S.nsym * nki * per);
  for (int64_t i = 0; i < S.nsym * nki; ++i)
    CQ_CHECK_CUDA(cudaMemcpyAsync(S.Xs.p + i * per, c->X.p + S.ks_lex[i] * per,
                                  per * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  S.Xibz.ensure((size_t)nki * per);
  for (int64_t i = 0; i < nki; ++i)
    CQ_CHECK_CUDA(cudaMemcpyAsync(S.Xibz.p + i * per, c->X.p + S.lex[i] * per,
                                  per * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  S.Li.ensure((size_t)nqi * pp);
  S.LHi.ensure((size_t)nqi * pp);
  S.Vi.ensure((size_t)nqi * pp);
  const bool mixed = (c->mode == COQUI_B200_MIXED);
  if (mixed) {
    S.Lci.ensure((size_t)nqi * pp);
    S.LHci.ensure((size_t)nqi * pp);
  }
  for (int64_t i = 0; i < nqi; ++i) {
    const int64_t q = S.q_lex[i];
    const size_t b = pp * sizeof(double2);
    CQ_CHECK_CUDA(cudaMemcpyAsync(S.Li.p + i * pp, c->L.p + q * pp, b, cudaMemcpyDeviceToDevice, c->st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(S.LHi.p + i * pp, c->LH.p + q * pp, b, cudaMemcpyDeviceToDevice, c->st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(S.Vi.p + i * pp, c->V.p + q * pp, b, cudaMemcpyDeviceToDevice, c->st));
    if (mixed) {
      const size_t bc = pp * sizeof(float2);
      CQ_CHECK_CUDA(cudaMemcpyAsync(S.Lci.p + i * pp, c->Lc.p + q * pp, bc, cudaMemcpyDeviceToDevice, c->st));
      CQ_CHECK_CUDA(cudaMemcpyAsync(S.LHci.p + i * pp, c->LHc.p + q * pp, bc, cudaMemcpyDeviceToDevice, c->st));
    }
  }
  if (mixed) cq::tc_pack_X(S.Xtc, S.Xs.p, S.nsym * nki, Np, nb, c->st);
  CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
  S.thc_ready = true;
}

// G on the IBZ k-points (host) -> the unfolded G of every k-point in c->G
void sym_upload_g(Ctx* c, const double* G_tskij) {
  SymState& S = *c->sym;
  CQ_REQUIRE(G_tskij, COQUI_B200_EINVAL, "the IBZ path needs G_tskij (no resident G)");
  const int64_t nb = c->nb, nki = S.nk_ibz;
  const size_t n = (size_t)c->nt * nki * nb * nb;
  S.Gi.ensure(n);
  upload(c, S.Gi.p, G_tskij, n * sizeof(double2));
  c->G.ensure((size_t)c->nt * c->nk * nb * nb);
  cq::launch_unfold_g(S.Gi.p, c->G.p, S.unfold.p, c->nt, c->nk, nki, nb, c->st);
  c->g_resident = false;
  c->g_pipelined = false;
  c->gcache_valid = false;
}

// Pi(tau) on the IBZ q-points into S.PWi (nth, nq_ibz, Np, Np)
void sym_pi(Ctx* c) {
  SymState& S = *c->sym;
  eval_pi_device(c);
  c->mark("EVALUATE_PI_R");
  const int64_t pp = c->Np * c->Np;
  S.PWi.ensure((size_t)c->nmax * S.nq_ibz * pp * c->elem());
  if (c->mode == COQUI_B200_FP64)
    cq::launch_gather_transpose<double>((const double2*)c->PW.p, (double2*)S.PWi.p, S.qsrc.p,
                                        c->nth, c->nq, S.nq_ibz, c->Np, c->st);
  else
    cq::launch_gather_transpose<float>((const float2*)c->PW.p, (float2*)S.PWi.p, S.qsrc.p, c->nth,
                                       c->nq, S.nq_ibz, c->Np, c->st);
  c->mark("PI_IBZ");
  S.w_valid = false;
}

// Dyson step of every (iW, q_ibz) problem on S.PWi
void sym_dyson(Ctx* c, bool want_w, bool want_e, std::vector<double>* ld,
               std::vector<double2>* tr) {
  SymState& S = *c->sym;
  cq::DysonArgs a;
  a.Np = c->Np;
  a.nq = S.nq_ibz;
  a.nw = c->nwh;
  a.L = S.Li.p;
  a.LH = S.LHi.p;
  a.V = S.Vi.p;
  a.Lc = S.Lci.p;
  a.LHc = S.LHci.p;
  a.want_w = want_w;
  a.want_e = want_e;
  a.mixed = (c->mode == COQUI_B200_MIXED);
  a.PW = S.PWi.p;
  a.prof = &c->prof;
  const int64_t nprob = c->nwh * S.nq_ibz;
  c->dinfo.ensure(nprob);
  c->dlogdet.ensure(nprob);
  c->dtrace.ensure(nprob);
  a.info = c->dinfo.p;
  a.logdet = c->dlogdet.p;
  a.trace = c->dtrace.p;
  cq::dyson_run(a, c->dyn, c->st, ld, tr);
}

void sym_update_w(Ctx* c) {
  SymState& S = *c->sym;
  sym_prepare_thc(c);
  sym_pi(c);
  const int64_t ncol = S.nq_ibz * c->Np * c->Np;
  ir_apply(c, S.PWi.p, ncol, (int)c->nth, (int)c->nwh, c->dTwt.p);
  c->mark("IMAG_FT_TtoW");
  sym_dyson(c, true, false, nullptr, nullptr);
  c->mark("EVALUATE_W");
  ir_apply(c, S.PWi.p, ncol, (int)c->nwh, (int)c->nth, c->dTtw.p);
  c->mark("IMAG_FT_WtoT");
  S.w_valid = true;
  c->w_valid = false;
}

// Sigma_ab = X^H S X for nkx problems with the given X (FP64 form)
void a2p_with(Ctx* c, const double2* X, int64_t nkx, const double2* Sk, double2* out) {
  const int64_t nb = c->nb, Np = c->Np;
  c->Tproj.ensure((size_t)nkx * Np * nb);
  zgemm_rm(c, 'C', 'N', nb, Np, Np, make_double2(1, 0), X, nb, Np * nb, Sk, Np, Np * Np,
           make_double2(0, 0), c->Tproj.p, Np, Np * nb, nkx);
  zgemm_rm(c, 'N', 'N', nb, nb, Np, make_double2(1, 0), c->Tproj.p, Np, Np * nb, X, nb,
           Np * nb, make_double2(0, 0), out, nb, nb * nb, nkx);
}

bool sym_div_active(const Ctx* c) { return c->div != 0 && c->sym->nq_ibz > 1; }

// eps_inv_head_t over Qpts_ibz (g0_div_utils.hpp:55-111, 180-214): eps^-1 per (tau, q_ibz) of
// the IBZ W, then the head of the treatment in effect into c->head_h (and out, if not null)
void sym_eps_head(Ctx* c, double* out) {
  SymState& S = *c->sym;
  cq::Prof::Scope sc(&c->prof, "eps_head");
  CQ_REQUIRE(S.w_valid, COQUI_B200_EINVAL, "no screened interaction: call update_w or set_w");
  const int64_t nqi = S.nq_ibz, Np = c->Np, nth = c->nth;
  S.chi_i.ensure((size_t)nqi * Np);
  S.fac_i.ensure((size_t)nqi);
  std::vector<double> qn(nqi), qz(nqi);
  int64_t qsm = 0;
  double best = -1;
  for (int64_t i = 0; i < nqi; ++i) {
    const int64_t q = S.q_lex[i];
    CQ_CHECK_CUDA(cudaMemcpyAsync(S.chi_i.p + i * Np, c->chi.p + q * Np, Np * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, c->st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(S.fac_i.p + i, c->fac.p + q, sizeof(double),
                                  cudaMemcpyDeviceToDevice, c->st));
    qn[i] = c->qnorm[q];
    qz[i] = c->qz[q];
    if (nqi > 1 && qn[i] > 0.0 && (best < 0 || qn[i] < best)) {  // find_smallest_qabs
      best = qn[i];
      qsm = i;
    }
  }
  c->eps.ensure((size_t)nth * nqi);
  if (c->mode == COQUI_B200_FP64)
    cq::launch_eps_head<double>((const double2*)S.PWi.p, S.chi_i.p, S.fac_i.p, c->eps.p, nth, nqi,
                                Np, c->st);
  else
    cq::launch_eps_head<float>((const float2*)S.PWi.p, S.chi_i.p, S.fac_i.p, c->eps.p, nth, nqi,
                               Np, c->st);
  S.eps_i.resize((size_t)nth * nqi);
  download(c, S.eps_i.data(), c->eps.p, S.eps_i.size() * sizeof(double2));
  CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
  select_head_from(c, S.eps_i, nqi, qn, qz, qsm);
  if (out)
    for (int64_t t = 0; t < nth; ++t) {
      out[2 * t] = c->head_h[t].x;
      out[2 * t + 1] = c->head_h[t].y;
    }
}

// eval_Sigma_all_kspace for t and beta - t into c->Sig (nt, nk_ibz, nb, nb).  Per tau slice:
// one gather pass forms the Sigma_PQ rows of every (isym, ik), one batched projection takes
// them to the orbitals at ks_to_k, D^H Sigma_ab D per row, and the rows of each ik are summed.
void sym_sigma(Ctx* c, double* host_out) {
  SymState& S = *c->sym;
  CQ_REQUIRE(S.w_valid, COQUI_B200_EINVAL, "no screened interaction: call update_w or set_w");
  sym_prepare_thc(c);
  const int64_t nt = c->nt, nth = c->nth, nk = c->nk, nb = c->nb, Np = c->Np;
  const int64_t nki = S.nk_ibz, nqi = S.nq_ibz, pp = Np * Np, bb = nb * nb;
  const int64_t nrow = S.nsym * nki;
  const size_t es = c->elem(), slab = (size_t)nk * pp * es;
  c->Gp.ensure(slab);
  S.Sq.ensure((size_t)nrow * pp * es);
  S.Sab.ensure((size_t)nrow * bb);
  S.Tab.ensure((size_t)nrow * bb);
  S.Rab.ensure((size_t)nrow * bb);
  c->Sig.ensure((size_t)nt * nki * bb);
  CQ_CHECK_CUDA(cudaMemsetAsync(c->Sig.p, 0, (size_t)nt * nki * bb * sizeof(double2), c->st));
  // G_PQ of every tau is still in the cache when the polarizability of this G just ran
  unsigned char* cache = c->gcache_valid ? c->Gcache.p : nullptr;
  c->gcache_valid = false;
  const double factor = -1.0 / (double)nk;
  const bool fp64 = (c->mode == COQUI_B200_FP64);
  for (int64_t it = 0; it < nth; ++it) {
    for (int minus = 0; minus < 2; ++minus) {
      const int64_t itg = minus ? nt - it - 1 : it;
      if (minus && itg == nth - 1) continue;  // odd nt: the middle slice once (thc_gw.icc:297)
      const unsigned char* g = c->Gp.p;
      if (cache && gcached(c, itg))
        g = gslab(c, itg);
      else
        project_p2a(c, c->G.p + itg * nk * bb, c->Gp.p);
      const unsigned char* W = S.PWi.p + (size_t)it * nqi * pp * es;
      {
        cq::Prof::Scope sc(&c->prof, "sigma_ksum");
        if (fp64)
          cq::launch_sigma_ksum<double>((const double2*)g, (const double2*)W, S.terms.p, S.rows.p,
                                        nrow, nk, nqi, pp, factor, (double2*)S.Sq.p, c->st);
        else
          cq::launch_sigma_ksum<float>((const float2*)g, (const float2*)W, S.terms.p, S.rows.p,
                                       nrow, nk, nqi, pp, factor, (float2*)S.Sq.p, c->st);
      }
      {
        cq::Prof::Scope sc(&c->prof, "proj_a2p", nrow);
        if (fp64)
          a2p_with(c, S.Xs.p, nrow, (const double2*)S.Sq.p, S.Sab.p);
        else
          cq::tc_project_a2p(S.Xtc, (const float2*)S.Sq.p, S.Sab.p, nrow, Np, nb, nrow, c->st);
      }
      // D^H Sigma_ab D per (isym, ik) (the identity operation's D is the identity), then the
      // rows of each ik summed into Sigma(itg, ik)
      zgemm_rm(c, 'C', 'N', nb, nb, nb, make_double2(1, 0), S.D.p, nb, bb, S.Sab.p, nb, bb,
               make_double2(0, 0), S.Tab.p, nb, bb, nrow);
      zgemm_rm(c, 'N', 'N', nb, nb, nb, make_double2(1, 0), S.Tab.p, nb, bb, S.D.p, nb, bb,
               make_double2(0, 0), S.Rab.p, nb, bb, nrow);
      cq::launch_add_blocks(S.Rab.p, c->Sig.p + itg * nki * bb, S.nsym, nki * bb, c->st);
    }
  }
  // Sigma_div_correction on the IBZ k-points (thc_gw.icc:31-33, 446-526)
  if (sym_div_active(c)) {
    CQ_REQUIRE(c->chi0c.n >= (size_t)Np, COQUI_B200_EINVAL,
               "the gygi treatments of Sigma need chi_head (coqui_b200_set_div_treatment)");
    sym_eps_head(c, nullptr);
    bool fresh = false;  // T^k from the current X and chi_head
    sigma_div_correction_on(c, nki, S.Xibz.p, S.Gi.p, c->Sig.p, S.Tdiv, fresh);
  }
  c->mark("EVALUATE_SIGMA_K");
  if (host_out) {
    download(c, host_out, c->Sig.p, (size_t)nt * nki * bb * sizeof(double2));
    c->mark("d2h_Sigma");
  }
}

void sym_eval_pi(Ctx* c, const double* G_tskij, double* Pi_tqPQ) {
  SymState& S = *c->sym;
  c->begin_timing();
  sym_upload_g(c, G_tskij);
  c->mark("h2d_G");
  sym_pi(c);
  if (Pi_tqPQ) {
    const int64_t slab = S.nq_ibz * c->Np * c->Np;
    if (c->mode == COQUI_B200_FP64) {
      download(c, Pi_tqPQ, S.PWi.p, (size_t)c->nth * slab * sizeof(double2));
    } else {
      c->stage.ensure(slab);
      for (int64_t t = 0; t < c->nth; ++t) {
        cq::launch_to_c128<float>((float2*)S.PWi.p + t * slab, c->stage.p, slab, c->st);
        download(c, Pi_tqPQ + 2 * t * slab, c->stage.p, slab * sizeof(double2));
      }
    }
    c->mark("d2h");
  }
  c->end_timing();
}

void sym_download_w(Ctx* c, double* dW_qtPQ) {
  SymState& S = *c->sym;
  const int64_t ncol = c->Np * c->Np, per_q = c->nth * ncol;
  c->stage.ensure(per_q);
  for (int64_t q = 0; q < S.nq_ibz; ++q) {
    if (c->mode == COQUI_B200_FP64)
      cq::launch_tq_to_qt_c128<double>((double2*)S.PWi.p, c->stage.p, c->nth, S.nq_ibz, ncol, q,
                                       1, c->st);
    else
      cq::launch_tq_to_qt_c128<float>((float2*)S.PWi.p, c->stage.p, c->nth, S.nq_ibz, ncol, q, 1,
                                      c->st);
    download(c, dW_qtPQ + 2 * q * per_q, c->stage.p, per_q * sizeof(double2));
  }
}

void sym_set_w(Ctx* c, const double* dW_qtPQ) {
  SymState& S = *c->sym;
  const int64_t ncol = c->Np * c->Np, n = S.nq_ibz * c->nth * ncol;
  S.PWi.ensure((size_t)c->nmax * S.nq_ibz * ncol * c->elem());
  c->stage.ensure(n);
  upload(c, c->stage.p, dW_qtPQ, n * sizeof(double2));
  if (c->mode == COQUI_B200_FP64)
    cq::launch_qt_to_tq<double>(c->stage.p, (double2*)S.PWi.p, c->nth, S.nq_ibz, ncol, c->st);
  else
    cq::launch_qt_to_tq<float>(c->stage.p, (float2*)S.PWi.p, c->nth, S.nq_ibz, ncol, c->st);
  CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
  c->stage.release();
  S.w_valid = true;
}

double sym_rpa_energy(Ctx* c, const double* G_tskij) {
  SymState& S = *c->sym;
  c->begin_timing();
  sym_upload_g(c, G_tskij);
  c->mark("h2d_G");
  sym_prepare_thc(c);
  sym_pi(c);
  ir_apply(c, S.PWi.p, S.nq_ibz * c->Np * c->Np, (int)c->nth, (int)c->nwh, c->dTwt.p);
  c->mark("IMAG_FT_TtoW");
  std::vector<double> ld;
  std::vector<double2> tr;
  sym_dyson(c, false, true, &ld, &tr);
  c->mark("EVALUATE_RPA");
  for (double v : ld)
    CQ_REQUIRE(std::isfinite(v), COQUI_B200_ENOTHPD, "I - Pi V is not positive definite");
  const double e = rpa_energy_from(c, ld, tr, S.qw);
  c->end_timing();
  return e;
}

}  // namespace

extern "C" int coqui_b200_set_symmetry(coqui_b200_ctx* c, const coqui_b200_symmetry* sym) {
  return guarded(c, [&] {
    if (!sym) {
      c->sym.reset();
      c->gcache_valid = false;
      c->g_resident = false;
      return;
    }
    CQ_REQUIRE(c->have_k, COQUI_B200_EINVAL, "set_kmesh not called");
    const coqui_b200_symmetry& m = *sym;
    const int64_t nk = c->nk, nq = c->nq, nb = c->nb;
    CQ_REQUIRE(m.k_lex && m.kp_to_ibz && m.kp_trev && m.kp_trev_pair && m.qp_to_ibz &&
                   m.qp_trev && m.qminus && m.nq_per_s && m.Qs && m.ks_to_k,
               COQUI_B200_EINVAL, "null symmetry map");
    CQ_REQUIRE(m.nk_ibz >= 1 && m.nk_ibz <= nk && m.nq_ibz >= 1 && m.nq_ibz <= nq &&
                   m.nsym >= 1 && m.ld_Qs >= 1,
               COQUI_B200_EINVAL, "symmetry sizes out of range");
    std::unique_ptr<SymState> S(new SymState());
    S->nk_ibz = m.nk_ibz;
    S->nq_ibz = m.nq_ibz;
    S->nsym = m.nsym;
    // k order: a permutation of the grid, IBZ points first and mapped to themselves
    S->lex.assign(m.k_lex, m.k_lex + nk);
    std::vector<int64_t> inv(nk, -1);
    for (int64_t i = 0; i < nk; ++i) {
      const int64_t p = S->lex[i];
      CQ_REQUIRE(p >= 0 && p < nk && inv[p] < 0, COQUI_B200_EINVAL,
                 "k_lex is not a permutation of the grid");
      inv[p] = i;
    }
    std::vector<int> unfold(nk);
    for (int64_t i = 0; i < nk; ++i) {
      const int64_t j = m.kp_to_ibz[i];
      const bool tr = m.kp_trev[i] != 0;
      CQ_REQUIRE(j >= 0 && j < m.nk_ibz, COQUI_B200_EINVAL, "kp_to_ibz out of range");
      if (i < m.nk_ibz)
        CQ_REQUIRE(j == i && !tr, COQUI_B200_EINVAL, "the IBZ k-points must come first");
      if (tr) {
        const int64_t p = m.kp_trev_pair[i];
        CQ_REQUIRE(p >= 0 && p < nk && !m.kp_trev[p] && m.kp_to_ibz[p] == j &&
                       S->lex[p] == lex_combine(c, 0, S->lex[i], -1),
                   COQUI_B200_EINVAL, "kp_trev_pair is not the -k partner without time reversal");
      }
      unfold[S->lex[i]] = (int)j | (tr ? (1 << 30) : 0);
    }
    // q maps (Qpts = kpts)
    S->qw.assign(m.nq_ibz, 0.0);
    for (int64_t q = 0; q < nq; ++q) {
      const int64_t j = m.qp_to_ibz[q];
      CQ_REQUIRE(j >= 0 && j < m.nq_ibz, COQUI_B200_EINVAL, "qp_to_ibz out of range");
      if (q < m.nq_ibz)
        CQ_REQUIRE(j == q && !m.qp_trev[q], COQUI_B200_EINVAL, "the IBZ q-points must come first");
      const int64_t mq = m.qminus[q];
      CQ_REQUIRE(mq >= 0 && mq < nq && S->lex[mq] == lex_combine(c, 0, S->lex[q], -1),
                 COQUI_B200_EINVAL, "qminus is not -q");
      S->qw[j] += 1.0;
    }
    std::vector<int> qsrc(m.nq_ibz);
    S->q_lex.resize(m.nq_ibz);
    for (int64_t i = 0; i < m.nq_ibz; ++i) {
      S->q_lex[i] = S->lex[i];
      qsrc[i] = (int)S->lex[m.qminus[i]];
    }
    // self-energy terms per (isym, ik), thc_gw.icc:366-401
    std::vector<char> seen(nq, 0);
    std::vector<int4> terms;
    S->ks_lex.resize(m.nsym * m.nk_ibz);
    for (int64_t s = 0; s < m.nsym; ++s) {
      const int64_t nqs = m.nq_per_s[s];
      CQ_REQUIRE(nqs >= 0 && nqs <= m.ld_Qs, COQUI_B200_EINVAL, "nq_per_s out of range");
      S->nterm.push_back(nqs);
      S->term_off.push_back(terms.size());
      for (int64_t j = 0; j < nqs; ++j) {
        const int64_t qp = m.Qs[s * m.ld_Qs + j];
        CQ_REQUIRE(qp >= 0 && qp < nq && !seen[qp], COQUI_B200_EINVAL,
                   "Qs must list every q-point exactly once");
        seen[qp] = 1;
      }
      for (int64_t ik = 0; ik < m.nk_ibz; ++ik) {
        const int64_t ks = m.ks_to_k[s * nk + ik];
        CQ_REQUIRE(ks >= 0 && ks < nk, COQUI_B200_EINVAL, "ks_to_k out of range");
        S->ks_lex[s * m.nk_ibz + ik] = S->lex[ks];
        for (int64_t j = 0; j < nqs; ++j) {
          const int64_t qp = m.Qs[s * m.ld_Qs + j];
          const int64_t qs = m.qp_to_ibz[qp];
          const bool qtr = m.qp_trev[qp] != 0;
          // ks - qs, or ks - (-qs) = ks + qs for a time-reversal q-point (qk_to_k2)
          const int64_t km = inv[lex_combine(c, S->lex[ks], S->lex[qs], qtr ? +1 : -1)];
          const bool ktr = m.kp_trev[km] != 0;
          const int64_t kg = ktr ? m.kp_trev_pair[km] : km;
          terms.push_back(make_int4((int)qs, (int)S->lex[kg], (ktr ? 1 : 0) | (qtr ? 2 : 0), 0));
        }
      }
    }
    for (int64_t q = 0; q < nq; ++q)
      CQ_REQUIRE(seen[q], COQUI_B200_EINVAL, "Qs must list every q-point exactly once");
    // rotations d[isym, k]: identity for the identity operation or when not given
    const int64_t bb = nb * nb;
    S->D_h.assign((size_t)m.nsym * m.nk_ibz * bb, make_double2(0, 0));
    for (int64_t s = 0; s < m.nsym; ++s)
      for (int64_t ik = 0; ik < m.nk_ibz; ++ik) {
        double2* d = S->D_h.data() + (s * m.nk_ibz + ik) * bb;
        if (s == 0 || !m.D) {
          for (int64_t a = 0; a < nb; ++a) d[a * nb + a] = make_double2(1, 0);
        } else {
          const double* src = m.D + 2 * (s * m.nk_ibz + ik) * bb;
          for (int64_t e = 0; e < bb; ++e) {
            CQ_REQUIRE(std::isfinite(src[2 * e]) && std::isfinite(src[2 * e + 1]),
                       COQUI_B200_EINVAL, "D holds NaN or Inf values");
            d[e] = make_double2(src[2 * e], src[2 * e + 1]);
          }
        }
      }
    S->unfold.ensure(nk);
    upload(c, S->unfold.p, unfold.data(), nk * sizeof(int));
    S->qsrc.ensure(m.nq_ibz);
    upload(c, S->qsrc.p, qsrc.data(), m.nq_ibz * sizeof(int));
    std::vector<int2> rows;
    for (int64_t s = 0; s < m.nsym; ++s)
      for (int64_t ik = 0; ik < m.nk_ibz; ++ik)
        rows.push_back(make_int2((int)(S->term_off[s] + ik * S->nterm[s]), (int)S->nterm[s]));
    CQ_REQUIRE(terms.size() < (size_t)0x7fffffff, COQUI_B200_EUNSUPPORTED,
               "too many self-energy terms");
    S->terms.ensure(std::max<size_t>(1, terms.size()));
    if (!terms.empty()) upload(c, S->terms.p, terms.data(), terms.size() * sizeof(int4));
    S->rows.ensure(rows.size());
    upload(c, S->rows.p, rows.data(), rows.size() * sizeof(int2));
    S->D.ensure(S->D_h.size());
    upload(c, S->D.p, S->D_h.data(), S->D_h.size() * sizeof(double2));
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->sym = std::move(S);
    c->gcache_valid = false;
    c->g_resident = false;
    c->w_valid = false;
  });
}
