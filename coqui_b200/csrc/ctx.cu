// C ABI of the THC-RPA/GW hot path: context, data upload and the solver entry points.
//
// Pipeline of one screened-interaction update (scr_coulomb_t::update_w,
// src/methods/scr_coulomb/scr_coulomb_t.cpp:37-95), all on one stream:
//   for tau in [0, nt_half): G^k_PQ(tau), G^k_PQ(beta - tau)  (projection GEMMs)
//                            -> fused k->R DFT, -2 Gp o conj(Gn), R->q DFT -> Pi(tau)
//   Pi(tau) -> Pi(iW)  (in-place IR transform)
//   per (q, iW): V = L L^H, M = L^H Pi L, I - M = C C^H (FP64), W = Y^H Y - V, Y = C^{-1} L^H
//   W(iW) -> W(tau)    (in-place IR transform), eps^-1 head.
// The self-energy and the RPA energy reuse the same stages.
#include <algorithm>
#include <complex>
#include <cstring>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "chol.cuh"
#include "dyson.cuh"
#include "kernels.cuh"
#include "mlp.cuh"
#include "scgw.cuh"
#include "sym.cuh"
#include "tc_gemm.cuh"
#include "zgemm.cuh"

using cq::Error;
using cq::KGrid;

namespace {

const char* kVersion = "coqui_b200 0.1.0 (sm_100a)";

using cq::DevBuf;

}  // namespace

// Symmetry-reduced k-space path (coqui_b200_set_symmetry): the mean field's maps translated to
// lexicographic k positions, the per-symmetry self-energy term lists, and the IBZ buffers.
struct SymState {
  int64_t nk_ibz = 0, nq_ibz = 0, nsym = 0;
  std::vector<int64_t> lex;       // the reference's k index -> lexicographic position
  std::vector<int64_t> ks_lex;    // (nsym, nk_ibz) lexicographic position of ks_to_k
  std::vector<int64_t> q_lex;     // (nq_ibz) lexicographic position of the IBZ q-points
  std::vector<double> qw;         // (nq_ibz) number of 1st-BZ q-points mapped to each
  std::vector<int64_t> nterm;     // (nsym) self-energy terms per IBZ k-point (nq_per_s)
  std::vector<size_t> term_off;   // (nsym) offset of the isym block in terms
  std::vector<double2> D_h;       // (nsym, nk_ibz, nb, nb), block 0 the identity
  DevBuf<int> unfold;             // (nk) lexicographic k -> IBZ index | time reversal << 30
  DevBuf<int> qsrc;               // (nq_ibz) lexicographic position of -q
  DevBuf<int4> terms;             // (w slab, G slab, conj flags) per (isym, ik, term)
  DevBuf<int2> rows;              // (nsym * nk_ibz): (first term, term count)
  DevBuf<double2> D;
  // built from the THC data on first use (set_thc clears thc_ready)
  bool thc_ready = false;
  DevBuf<double2> Xs;             // (nsym, nk_ibz, Np, nb): X at ks_to_k(isym, ik)
  cq::TcOperand Xtc;              // mixed form: Xs packed for the tensor-core projection
  DevBuf<double2> Li, LHi, Vi;    // (nq_ibz, Np, Np) at the IBZ q-points
  DevBuf<float2> Lci, LHci;
  DevBuf<double2> Gi;             // (nt, nk_ibz, nb, nb) G on the IBZ k-points
  DevBuf<unsigned char> PWi;      // (nmax, nq_ibz, Np, Np) Pi / W on the IBZ q-points
  DevBuf<unsigned char> Sq;       // (nsym, nk_ibz, Np, Np) Sigma_PQ rows of one tau
  DevBuf<double2> Sab, Tab, Rab;  // (nsym, nk_ibz, nb, nb)
  // long-wavelength treatments on the IBZ: X of the IBZ k-points, chi-bar heads and prefactors
  // of the IBZ q-points, T^k of Sigma_div_correction, eps^-1 per (tau, q_ibz)
  DevBuf<double2> Xibz, chi_i, Tdiv;
  DevBuf<double> fac_i;
  std::vector<double2> eps_i;
  bool w_valid = false;
};

struct coqui_b200_ctx {
  coqui_b200_dims d{};
  int64_t ns = 1, nk = 0, nq = 0, nb = 0, Np = 0, nt = 0, nth = 0, nwb = 0, nwh = 0, nmax = 0;
  KGrid g{1, 1, 1};
  int mode = COQUI_B200_MIXED;
  int dev = 0;
  std::string err;
  cudaStream_t st = nullptr;
  int64_t launch_base = 0;
  bool have_ir = false, have_k = false, have_thc = false, w_valid = false, w_in_R = false;
  bool g_resident = false;
  cq::Prof prof;
  std::unique_ptr<SymState> sym;  // set: the IBZ k-space path

  // host-side IR data
  std::vector<double2> Twt_pos, Ttw_pos, Ttw_bb, T_beta;
  // host-side head factors
  std::vector<double> head_fac;
  int64_t q_smallest = 0;

  // device data
  DevBuf<double2> X, V, L, LH, chi, G, Sig, Tproj, stage, dTwt, dTtw;
  DevBuf<double> dTwtR, dTtwR;  // real parts, used when the PH matrices are real
  bool ir_real = false;
  DevBuf<double> fac;
  DevBuf<double2> eps;
  DevBuf<unsigned char> Gp, Gn, PW;  // storage precision, bytes
  DevBuf<unsigned char> dyn;         // Dyson scratch
  DevBuf<float2> Lc, LHc;            // complex64 L, L^H for the tensor-core Dyson products
  cq::TcOperand Xtc;                 // packed X for the tensor-core projections
  DevBuf<double2> Gx;                // primary_to_aux staging (the resident G stays intact)

  // G_PQ(tau) for every tau, computed by the polarizability and reused (then overwritten in
  // place) by the self-energy of the same G; allocated when it fits in half the free memory
  DevBuf<unsigned char> Gcache;
  bool gcache_valid = false;
  // tau pairs the cache holds: slices [0, gcache_pairs) and [nt - gcache_pairs, nt); all nt
  // slices (indexed by tau) when gcache_pairs == nth
  int64_t gcache_pairs = 0;
  int64_t gcache_limit = -1;  // bytes; -1: half the free memory at first use

  // Dyson results per (iW, q) problem on the device
  DevBuf<int> dinfo;
  DevBuf<int> flag;  // input checks
  DevBuf<double> dlogdet;
  DevBuf<double2> dtrace;
  // CUDA graph of the resident-G GW iteration (captured on the first of consecutive calls)
  bool capturing = false;
  // host buffers baked into the captured graph (nullptr: resident G / Sigma left on the device)
  const double* graph_g = nullptr;
  double* graph_s = nullptr;
  // the Dyson step leaves its per-problem status on the device (checked after the iteration)
  bool defer_dyson_check = false;
  cudaGraphExec_t gexec = nullptr;
  int64_t calls = 0, graph_call = -2, graph_launches = 0;
  // the same for the RPA energy (polarizability, tau -> w, factorisations)
  cudaGraphExec_t rexec = nullptr;
  const double* rgraph_g = nullptr;
  int64_t rgraph_call = -2, rgraph_launches = 0;

  // self-consistent loop: fermionic IR grid, mean field, iteration state
  bool have_irf = false, have_mf = false;
  int64_t nwf = 0;
  double beta = 0, mu = 0;
  std::vector<int64_t> wnf;
  std::vector<double2> Ttw_ff_h;           // (nt, nwf)
  DevBuf<int64_t> dwnf;
  DevBuf<double2> dTwt_ff, dTtw_ff;        // (nwf, nt), (nt, nwf)
  DevBuf<double2> H0, Sov, F, F_mf, Dm;    // (nk, nb, nb)
  DevBuf<double2> Gw, Sw, Xw;              // (nwf, nk, nb, nb)
  DevBuf<double2> Gin;                     // G(tau) that produced the current Sigma
  DevBuf<double2> FS, prevFS;              // this / the previous iteration's (F, Sigma)
  DevBuf<int> ginfo;
  DevBuf<double> red;
  DevBuf<double2> trc;
  // long-wavelength treatment (div_treatment_e): 0 ignore_g0, 1 gygi, 2 gygi_extrplt,
  // 3 gygi_extrplt_2d; the madelung constant; conj(basis_head) at q = 0 (device)
  int div = 0;
  double madelung = 0;
  std::vector<double> qnorm, qz;   // |q| (as the reference forms it) and q_z per q-point
  DevBuf<double2> chi0c, Tdiv, divY;
  bool tdiv_valid = false;
  // eps^-1 head per (tau, q) of the current W (host, (nth, nq)) and the selected head (nth)
  std::vector<double2> eps_raw, head_h;
  bool eps_raw_valid = false;
  DevBuf<double> divf;
  DevBuf<const double2*> divp;     // pointer arrays of the batched correction products
  std::vector<const double2*> divp_h;
  // THC Hartree-Fock: bare V(q) transformed to R in FP64 (built on first use), scratch, and
  // whether the loop re-evaluates F = J + K from the density matrix
  DevBuf<double2> VR;
  bool vr_valid = false;
  DevBuf<double2> hfd, hfs, hff, hfv, hft, hfp;
  bool hf_on = false;
  int hf_div = 0;
  double hf_madelung = 0;
  int iter_alg = 0;                        // 0 damping, 1 commutator DIIS
  double mixing = 0.7;
  int64_t max_subsp = 5, diis_start = 5;
  std::vector<std::unique_ptr<DevBuf<double2>>> dx;  // DIIS x-vectors (F then Sigma)
  std::vector<std::unique_ptr<DevBuf<double2>>> dr;  // DIIS residuals (Sigma part)
  std::vector<std::complex<double>> dB;              // residual overlaps (row-major nB x nB)
  // learned update of the damped loop
  coqui_b200_mlp* mlp = nullptr;
  bool mlp_on = false, last_mlp = false;
  double mlp_max_jump = 5.0, r_prev = 0;
  int cooldown = 0;
  int64_t nhist = 0;
  DevBuf<double2> dhist;       // (4, nwf * nk * nb) diag Sigma_in(i w), oldest first
  DevBuf<double2> plain_saved; // the damped Sigma that the last proposal replaced
  DevBuf<double2> dtmp;        // (max(nt, nwf), nk * nb)

  // pipelined host transfers: G arrives in tau chunks on the copy stream (one event per
  // chunk) and Sigma leaves chunk by chunk while later chunks are computed
  cudaStream_t cs = nullptr;
  cudaEvent_t ev_st = nullptr;  // compute stream -> copy stream ordering
  std::vector<cudaEvent_t> up_ev;
  bool g_pipelined = false;

  // phase timing of the last call
  std::vector<std::pair<std::string, cudaEvent_t>> marks;
  std::vector<std::pair<std::string, double>> last_ms;

  size_t elem() const { return mode == COQUI_B200_FP64 ? sizeof(double2) : sizeof(float2); }

  void mark(const char* name) {
    if (capturing) return;  // the phases of a captured iteration are not recorded
    cudaEvent_t e;
    CQ_CHECK_CUDA(cudaEventCreate(&e));
    CQ_CHECK_CUDA(cudaEventRecord(e, st));
    marks.emplace_back(name, e);
  }
  void begin_timing() {
    for (auto& m : marks) cudaEventDestroy(m.second);
    marks.clear();
    mark("start");
  }
  void end_timing() {
    CQ_CHECK_CUDA(cudaStreamSynchronize(st));
    prof.resolve();
    last_ms.clear();
    for (size_t i = 1; i < marks.size(); ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, marks[i - 1].second, marks[i].second);
      last_ms.emplace_back(marks[i].first, ms);
    }
    for (auto& m : marks) cudaEventDestroy(m.second);
    marks.clear();
  }
};

namespace {

using Ctx = coqui_b200_ctx;

// After an error: let queued work and host copies finish before returning to the caller,
// whose host buffers they may still reference.
void settle(Ctx* c) {
  if (c->st) (void)cudaStreamSynchronize(c->st);
  if (c->cs) (void)cudaStreamSynchronize(c->cs);
}

template <typename F> int guarded(Ctx* c, F&& f) {
  if (!c) return COQUI_B200_EINVAL;
  ++c->calls;  // a captured iteration graph is replayed only by directly consecutive calls
  try {
    CQ_CHECK_CUDA(cudaSetDevice(c->dev));
    f();
    if (c->st) CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    if (c->cs) CQ_CHECK_CUDA(cudaStreamSynchronize(c->cs));
    if (cq::tc_take_nonfinite())
      throw Error(COQUI_B200_EINVAL, "G holds NaN or Inf values");
    if (cq::tc_take_error())
      throw Error(COQUI_B200_ETIMEDOUT, "a tensor-core kernel gave up a bounded wait");
    c->err.clear();
    return COQUI_B200_OK;
  } catch (const Error& e) {
    c->err = e.what();
    settle(c);
    // a non-finite G is the cause of whatever failed downstream of it (a factorisation without
    // positive pivots, say): report it as such
    bool nonfinite = false;
    try {
      nonfinite = cq::tc_take_nonfinite() != 0;
    } catch (const Error&) {
    }
    if (nonfinite) {
      c->err = "G holds NaN or Inf values";
      return COQUI_B200_EINVAL;
    }
    return e.code;
  } catch (const std::bad_alloc&) {
    c->err = "host allocation failed";
    settle(c);
    return COQUI_B200_ENOMEM;
  } catch (const std::exception& e) {
    c->err = e.what();
    settle(c);
    return COQUI_B200_EINVAL;
  }
}

// Row-major complex128 GEMM on the FP64 tensor cores (zgemm.cu): C = alpha op(A) op(B) +
// beta C, batched with constant strides (0 broadcasts an operand).
void zgemm_rm(Ctx* c, char opA, char opB, int64_t M, int64_t N, int64_t K, double2 alpha,
              const double2* A, int64_t lda, int64_t sA, const double2* B, int64_t ldb,
              int64_t sB, double2 beta, double2* C, int64_t ldc, int64_t sC, int64_t batch) {
  cq::ZgemmArgs z;
  z.opA = opA;
  z.opB = opB;
  z.M = M;
  z.N = N;
  z.K = K;
  z.alpha = alpha;
  z.beta = beta;
  z.A = A;
  z.lda = lda;
  z.sA = sA;
  z.B = B;
  z.ldb = ldb;
  z.sB = sB;
  z.C = C;
  z.ldc = ldc;
  z.sC = sC;
  z.batch = batch;
  cq::zgemm(z, c->st);
}

// The same with per-problem operand pointers (device arrays of batch pointers each).
void zgemm_rm_ptrs(Ctx* c, char opA, char opB, int64_t M, int64_t N, int64_t K, double2 alpha,
                   const double2* const* A, int64_t lda, const double2* const* B, int64_t ldb,
                   double2 beta, double2* const* C, int64_t ldc, int64_t batch) {
  cq::ZgemmArgs z;
  z.opA = opA;
  z.opB = opB;
  z.M = M;
  z.N = N;
  z.K = K;
  z.alpha = alpha;
  z.beta = beta;
  z.Ap = A;
  z.lda = lda;
  z.Bp = B;
  z.ldb = ldb;
  z.Cp = C;
  z.ldc = ldc;
  z.batch = batch;
  cq::zgemm(z, c->st);
}

void upload(Ctx* c, void* dst, const void* src, size_t bytes) {
  CQ_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->st));
}
void download(Ctx* c, void* dst, const void* src, size_t bytes) {
  CQ_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->st));
}

void require_ready(Ctx* c, bool thc, bool ir, bool k) {
  CQ_REQUIRE(!thc || c->have_thc, COQUI_B200_EINVAL, "set_thc not called");
  CQ_REQUIRE(!ir || c->have_ir, COQUI_B200_EINVAL, "set_ir not called");
  CQ_REQUIRE(!k || c->have_k, COQUI_B200_EINVAL, "set_kmesh not called");
}

// ---------------------------------------------------------------------------------------
// projections: O_PQ = X G X^H (primary -> aux) and O_ab = X^H O X (aux -> primary)
// ---------------------------------------------------------------------------------------

// ntau consecutive G slices (ntau, nk, nb, nb) complex128 on the device -> out (ntau, nk,
// Np, Np) in storage precision.  The tensor-core form batches all ntau * nk problems.
void p2a_fp64(Ctx* c, const double2* Gk, double2* out, int64_t ntau) {
  const int64_t nk = c->nk, nb = c->nb, Np = c->Np;
  c->Tproj.ensure((size_t)nk * Np * nb);
  for (int64_t t = 0; t < ntau; ++t) {
    const double2* G = Gk + t * nk * nb * nb;
    double2* O = out + t * nk * Np * Np;
    // T = X G  (Np x nb)
    zgemm_rm(c, 'N', 'N', Np, nb, nb, make_double2(1, 0), c->X.p, nb, Np * nb, G, nb, nb * nb,
             make_double2(0, 0), c->Tproj.p, nb, Np * nb, nk);
    // O = T X^H  (Np x Np)
    zgemm_rm(c, 'N', 'C', Np, Np, nb, make_double2(1, 0), c->Tproj.p, nb, Np * nb, c->X.p, nb,
             Np * nb, make_double2(0, 0), O, Np, Np * Np, nk);
  }
}
void a2p_fp64(Ctx* c, const double2* Sk, double2* out, int64_t ntau) {
  const int64_t nk = c->nk, nb = c->nb, Np = c->Np;
  c->Tproj.ensure((size_t)nk * Np * nb);
  for (int64_t t = 0; t < ntau; ++t) {
    const double2* S = Sk + t * nk * Np * Np;
    double2* O = out + t * nk * nb * nb;
    // T = X^H S  (nb x Np)
    zgemm_rm(c, 'C', 'N', nb, Np, Np, make_double2(1, 0), c->X.p, nb, Np * nb, S, Np, Np * Np,
             make_double2(0, 0), c->Tproj.p, Np, Np * nb, nk);
    // O = T X  (nb x nb)
    zgemm_rm(c, 'N', 'N', nb, nb, Np, make_double2(1, 0), c->Tproj.p, Np, Np * nb, c->X.p, nb,
             Np * nb, make_double2(0, 0), O, nb, nb * nb, nk);
  }
}

void project_p2a(Ctx* c, const double2* Gk, void* out, int64_t ntau = 1) {
  cq::Prof::Scope sc(&c->prof, "proj_p2a", ntau * c->nk);
  const int64_t nk = c->nk, nb = c->nb, Np = c->Np;
  if (c->mode == COQUI_B200_FP64) {
    p2a_fp64(c, Gk, (double2*)out, ntau);
  } else {
    cq::tc_project_p2a(c->Xtc, Gk, (float2*)out, nk, Np, nb, ntau * nk, c->st);
  }
}
// ntau consecutive slices (ntau, nk, Np, Np) in storage precision -> out (ntau, nk, nb, nb)
// complex128.
void project_a2p(Ctx* c, const void* Sk, double2* out, int64_t ntau = 1) {
  cq::Prof::Scope sc(&c->prof, "proj_a2p", ntau * c->nk);
  const int64_t nk = c->nk, nb = c->nb, Np = c->Np;
  if (c->mode == COQUI_B200_FP64) {
    a2p_fp64(c, (const double2*)Sk, out, ntau);
  } else {
    cq::tc_project_a2p(c->Xtc, (const float2*)Sk, out, nk, Np, nb, ntau * nk, c->st);
  }
}

// ---------------------------------------------------------------------------------------
// tau chunks: chunk i covers the tau pairs it in [a, b), i.e. the slices [a, b) and
// [nt - b, nt - a), in the order the polarizability consumes them (Pi(it) needs G(it) and
// G(nt - 1 - it), rpa_pi.icc:102-176).  At least 256 (tau, k) problems per chunk so that each
// batched projection fills the GPU.
// ---------------------------------------------------------------------------------------
int64_t tau_chunk(Ctx* c) {
  const int64_t want = (256 + c->nk - 1) / c->nk;
  return std::min<int64_t>(c->nth, std::max<int64_t>(4, want));
}
int64_t n_tau_chunks(Ctx* c) { return (c->nth + tau_chunk(c) - 1) / tau_chunk(c); }
void tau_chunk_range(Ctx* c, int64_t i, int64_t* a, int64_t* b) {
  *a = i * tau_chunk(c);
  *b = std::min<int64_t>(c->nth, *a + tau_chunk(c));
}

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// make the compute stream wait for the G slices of chunk i (pipelined upload only)
void wait_G_chunk(Ctx* c, int64_t i) {
  if (c->g_pipelined) CQ_CHECK_CUDA(cudaStreamWaitEvent(c->st, c->up_ev[(size_t)i], 0));
}

// Projected-G cache: every tau slice when nt slabs fit in half the free memory, else as many
// whole tau chunks (each a pair of slice ranges [a, b) and [nt - b, nt - a)) as fit, the
// first chunks; the polarizability fills it and the self-energy reuses it, projecting the
// slices outside it again.  nullptr when not even one chunk fits.  The size is fixed by the
// first allocation.
unsigned char* gcache(Ctx* c) {
  const size_t slab = (size_t)c->nk * c->Np * c->Np * c->elem();
  const size_t full = (size_t)c->nt * slab;
  const int64_t chunk = tau_chunk(c);
  const size_t pair = 2 * (size_t)chunk * slab;
  if (c->Gcache.n == 0) {
    size_t fr = 0, tot = 0;
    CQ_CHECK_CUDA(cudaMemGetInfo(&fr, &tot));
    // at most half the free memory, and the Dyson step keeps the memory for chunks of two
    // whole factorisation waves (fewer, smaller chunks cost it more than the cache saves)
    size_t budget = fr / 2;
    const size_t reserve =
        cq::dyson_reserve_bytes(c->Np, c->nwh * c->nq, c->mode != COQUI_B200_FP64);
    const size_t need = (reserve > c->dyn.n ? reserve - c->dyn.n : 0) + ((size_t)1 << 30);
    budget = std::min(budget, fr > need ? fr - need : 0);
    if (c->gcache_limit >= 0) budget = std::min(budget, (size_t)c->gcache_limit);
    if (full <= budget) {
      c->Gcache.ensure(full);
    } else {
      const int64_t nfit = std::min<int64_t>((int64_t)(budget / pair), n_tau_chunks(c) - 1);
      if (nfit <= 0) {
        c->gcache_pairs = 0;
        return nullptr;
      }
      c->Gcache.ensure((size_t)nfit * pair);
    }
  }
  if (c->Gcache.n >= full) {
    c->gcache_pairs = c->nth;
  } else {
    const int64_t nfit = std::min<int64_t>((int64_t)(c->Gcache.n / pair), n_tau_chunks(c) - 1);
    c->gcache_pairs = std::max<int64_t>(nfit, 0) * chunk;
  }
  return c->gcache_pairs > 0 ? c->Gcache.p : nullptr;
}

// whether the cache holds slice tau, and where
bool gcached(const Ctx* c, int64_t tau) {
  const int64_t A = c->gcache_pairs;
  return A >= c->nth || tau < A || tau >= c->nt - A;
}
unsigned char* gslab(Ctx* c, int64_t tau) {
  const size_t slab = (size_t)c->nk * c->Np * c->Np * c->elem();
  const int64_t A = c->gcache_pairs;
  const int64_t idx = (A >= c->nth || tau < A) ? tau : tau - c->nt + 2 * A;
  return c->Gcache.p + (size_t)idx * slab;
}
// whether tau chunk [a, b) lies in the cache (chunks are cached whole)
bool gchunk_cached(const Ctx* c, int64_t b) {
  return c->gcache_pairs >= c->nth || b <= c->gcache_pairs;
}

void eval_pi_device(Ctx* c) {
  const int64_t nk = c->nk, nb = c->nb, Np = c->Np, ncol = Np * Np, nt = c->nt;
  const size_t slab = (size_t)nk * ncol * c->elem();
  const size_t gsz = (size_t)nk * nb * nb;
  c->Gp.ensure(slab);
  c->Gn.ensure(slab);
  c->PW.ensure((size_t)c->nmax * c->nq * ncol * c->elem());
  unsigned char* cache = gcache(c);
  c->gcache_valid = false;
  const double sp = (c->ns == 2) ? -1.0 : -2.0;
  for (int64_t i = 0; i < n_tau_chunks(c); ++i) {
    int64_t a, b;
    tau_chunk_range(c, i, &a, &b);
    wait_G_chunk(c, i);
    const bool cached = cache && gchunk_cached(c, b);
    if (cached) {
      project_p2a(c, c->G.p + a * gsz, gslab(c, a), b - a);
      project_p2a(c, c->G.p + (nt - b) * gsz, gslab(c, nt - b), b - a);
    }
    for (int64_t it = a; it < b; ++it) {
      const unsigned char* gp = c->Gp.p;
      const unsigned char* gn = c->Gn.p;
      if (cached) {
        gp = gslab(c, it);
        gn = gslab(c, nt - it - 1);
      } else {
        project_p2a(c, c->G.p + it * gsz, c->Gp.p);
        project_p2a(c, c->G.p + (nt - it - 1) * gsz, c->Gn.p);
      }
      unsigned char* dst = c->PW.p + (size_t)it * c->nq * ncol * c->elem();
      cq::Prof::Scope sc(&c->prof, "pi_fused");
      if (c->mode == COQUI_B200_FP64)
        cq::launch_pi_fused<double>((const double2*)gp, (const double2*)gn, (double2*)dst, ncol,
                                    c->g, sp, c->st);
      else
        cq::launch_pi_fused<float>((const float2*)gp, (const float2*)gn, (float2*)dst, ncol, c->g,
                                   sp, c->st);
    }
  }
  c->gcache_valid = (cache != nullptr);
  c->w_valid = false;
}
// in-place tau <-> iW transform of buf (rows of ncol elements in storage precision)
void ir_apply(Ctx* c, unsigned char* buf, int64_t ncol, int n_in, int n_out, const double2* M) {
  cq::Prof::Scope sc(&c->prof, "ir_transform");
  if (c->ir_real) {
    const double* Mr = (M == c->dTwt.p) ? c->dTwtR.p : c->dTtwR.p;
    if (c->mode == COQUI_B200_FP64)
      cq::launch_ir_transform_real<double>((double2*)buf, ncol, n_in, n_out, Mr, c->st);
    else
      cq::launch_ir_transform_real<float>((float2*)buf, ncol, n_in, n_out, Mr, c->st);
    return;
  }
  if (c->mode == COQUI_B200_FP64)
    cq::launch_ir_transform<double>((double2*)buf, ncol, n_in, n_out, M, c->st);
  else
    cq::launch_ir_transform<float>((float2*)buf, ncol, n_in, n_out, M, c->st);
}
void ir_inplace(Ctx* c, int n_in, int n_out, const double2* M) {
  ir_apply(c, c->PW.p, c->nq * c->Np * c->Np, n_in, n_out, M);
}

void upload_G(Ctx* c, const double* G_tskij) {
  const size_t gsz = (size_t)c->nk * c->nb * c->nb;
  const size_t n = (size_t)c->nt * gsz;
  if (!G_tskij) {
    CQ_REQUIRE(c->g_resident, COQUI_B200_EINVAL, "G_tskij is null and no G is resident");
    return;
  }
  c->G.ensure(n);
  c->gcache_valid = false;
  c->g_resident = true;
  if (!is_pinned(G_tskij)) {
    c->g_pipelined = false;
    upload(c, c->G.p, G_tskij, n * sizeof(double2));
    return;
  }
  // page-locked source: copy chunk by chunk on the copy stream; the projections of chunk i
  // start once its event fired, while later chunks are still crossing the bus
  const int64_t nch = n_tau_chunks(c);
  while ((int64_t)c->up_ev.size() < nch) {
    cudaEvent_t e;
    CQ_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->up_ev.push_back(e);
  }
  CQ_CHECK_CUDA(cudaEventRecord(c->ev_st, c->st));  // earlier readers of the G buffer
  CQ_CHECK_CUDA(cudaStreamWaitEvent(c->cs, c->ev_st, 0));
  const double2* h = reinterpret_cast<const double2*>(G_tskij);
  for (int64_t i = 0; i < nch; ++i) {
    int64_t a, b;
    tau_chunk_range(c, i, &a, &b);
    const size_t bytes = (size_t)(b - a) * gsz * sizeof(double2);
    CQ_CHECK_CUDA(cudaMemcpyAsync(c->G.p + a * gsz, h + a * gsz, bytes, cudaMemcpyHostToDevice, c->cs));
    CQ_CHECK_CUDA(cudaMemcpyAsync(c->G.p + (c->nt - b) * gsz, h + (c->nt - b) * gsz, bytes,
                                  cudaMemcpyHostToDevice, c->cs));
    CQ_CHECK_CUDA(cudaEventRecord(c->up_ev[(size_t)i], c->cs));
  }
  c->g_pipelined = true;
}

// E_c accumulation (thc_rpa.icc:130-173) from per-(w, q) log det and traces; qw holds the
// q weights of the IBZ path (thc_rpa.icc:133), empty: every q-point once.
double rpa_energy_from(Ctx* c, const std::vector<double>& logdet, const std::vector<double2>& tr,
                       const std::vector<double>& qw = {}) {
  const int64_t nwb = c->nwb, nwh = c->nwh, nq = qw.empty() ? c->nq : (int64_t)qw.size();
  std::vector<std::complex<double>> e_w(nwb, 0.0);
  for (int64_t n = 0; n < nwh; ++n)
    for (int64_t q = 0; q < nq; ++q) {
      const int64_t p = n * nq + q;
      const double w = qw.empty() ? 1.0 : qw[q];
      const std::complex<double> v(w * (tr[p].x + logdet[p]), w * tr[p].y);
      const int64_t wn = nwb / 2 + n, mwn = nwb / 2 - n;
      e_w[wn] += v;
      if (mwn != wn) e_w[mwn] += v;
    }
  // e(tau) = Ttw_bb e(w) on the nt_f-point mesh, then tau -> beta^- with T_beta_t_ff
  std::complex<double> e = 0;
  for (int64_t t = 0; t < c->nt; ++t) {
    std::complex<double> et = 0;
    for (int64_t w = 0; w < nwb; ++w) {
      const double2 T = c->Ttw_bb[t * nwb + w];
      et += std::complex<double>(T.x, T.y) * e_w[w];
    }
    e += std::complex<double>(c->T_beta[t].x, c->T_beta[t].y) * et;
  }
  e /= (2.0 * (double)c->nk);
  return e.real();
}

}  // namespace

// ---------------------------------------------------------------------------------------
// self-consistent loop (scf_driver.cpp:90-173 for GW, hf = nullptr, constant mu)
// ---------------------------------------------------------------------------------------
// Fermionic IR transforms of n columns: out (nwf, n) = Twt_ff in (nt, n) and back.
void tau_to_w_ff(Ctx* c, const double2* in, double2* out, int64_t n) {
  zgemm_rm(c, 'N', 'N', c->nwf, n, c->nt, make_double2(1, 0), c->dTwt_ff.p, c->nt, 0, in, n, 0,
           make_double2(0, 0), out, n, 0, 1);
}
void w_to_tau_ff(Ctx* c, const double2* in, double2* out, int64_t n) {
  zgemm_rm(c, 'N', 'N', c->nt, n, c->nwf, make_double2(1, 0), c->dTtw_ff.p, c->nwf, 0, in, n, 0,
           make_double2(0, 0), out, n, 0, 1);
}

void require_scgw(Ctx* c) {
  require_ready(c, true, true, true);
  CQ_REQUIRE(c->have_irf, COQUI_B200_EINVAL, "set_ir_fermi not called");
  CQ_REQUIRE(c->have_mf, COQUI_B200_EINVAL, "set_mean_field not called");
}

// c->Dm <- -G(beta^-) of the resident G (IAFT.icc:226-238, simple_dyson.cpp:119-121), made
// Hermitian (scf_driver.cpp:140-143)
void dm_from_g(Ctx* c) {
  const int64_t ncol = c->nk * c->nb * c->nb;
  c->Dm.ensure(ncol);
  c->trc.ensure(c->nt);
  upload(c, c->trc.p, c->T_beta.data(), c->nt * sizeof(double2));
  zgemm_rm(c, 'N', 'N', 1, ncol, c->nt, make_double2(-1, 0), c->trc.p, c->nt, 0, c->G.p, ncol, 0,
           make_double2(0, 0), c->Dm.p, ncol, 0, 1);
  cq::hermitize_c128(c->Dm.p, c->nb, c->nk, c->st);
}

// simple_dyson.cpp:66-123 with the hermitization of scf_driver.cpp:140-143: c->G <- G(tau)
// from Sigma(tau) (device, (nt, nk, nb, nb)), c->Dm <- -G(beta^-).
void dyson_g_device(Ctx* c, const double2* Sig) {
  cq::Prof::Scope sc(&c->prof, "scgw_dyson_g");
  const int64_t nk = c->nk, nb = c->nb, ncol = nk * nb * nb, nw = c->nwf;
  c->Sw.ensure(nw * ncol);
  c->Xw.ensure(nw * ncol);
  c->ginfo.ensure(nw * nk);
  c->G.ensure(c->nt * ncol);
  c->Dm.ensure(ncol);
  tau_to_w_ff(c, Sig, c->Sw.p, ncol);
  cq::build_dyson_matrix(c->Sov.p, c->H0.p, c->F.p, c->Sw.p, c->Xw.p, c->dwnf.p, c->beta, c->mu,
                         nw, nk, nb, c->st);
  cq::invert_batched(c->Xw.p, nb, nw * nk, c->ginfo.p, c->st);
  w_to_tau_ff(c, c->Xw.p, c->G.p, ncol);
  dm_from_g(c);
  cq::hermitize_c128(c->G.p, nb, c->nt * nk, c->st);
  std::vector<int> info(nw * nk);
  CQ_CHECK_CUDA(cudaMemcpyAsync(info.data(), c->ginfo.p, info.size() * sizeof(int),
                                cudaMemcpyDeviceToHost, c->st));
  CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
  for (int v : info)
    CQ_REQUIRE(v == 0, COQUI_B200_ENOTHPD, "singular Dyson matrix (i w + mu) S - H0 - F - Sigma");
  // the resident G changed: no pipelined chunks, no cached projections
  c->g_resident = true;
  c->g_pipelined = false;
  c->gcache_valid = false;
}

// sum_k w_k sum_ij A_ij B_ji per leading index (w_k = 1/nk): out (nlead)
std::vector<std::complex<double>> k_traces(Ctx* c, const double2* A, const double2* B, int64_t nlead,
                                           int64_t b_mod) {
  const int64_t nk = c->nk, nb = c->nb;
  c->trc.ensure(nlead * nk);
  cq::trace_products(A, B, c->trc.p, nb, nlead * nk, b_mod, c->st);
  std::vector<double2> h(nlead * nk);
  CQ_CHECK_CUDA(cudaMemcpyAsync(h.data(), c->trc.p, h.size() * sizeof(double2),
                                cudaMemcpyDeviceToHost, c->st));
  CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
  std::vector<std::complex<double>> out(nlead, 0.0);
  for (int64_t l = 0; l < nlead; ++l)
    for (int64_t k = 0; k < nk; ++k)
      out[l] += std::complex<double>(h[l * nk + k].x, h[l * nk + k].y) / (double)nk;
  return out;
}

// Galitskii-Migdal energy (scf_common.cpp:87-136) of G(tau), Sigma(tau) on the device.
double gm_energy_device(Ctx* c, const double2* G, const double2* Sig) {
  cq::Prof::Scope sc(&c->prof, "scgw_energy");
  const int64_t ncol = c->nk * c->nb * c->nb, nw = c->nwf;
  c->Sw.ensure(nw * ncol);
  c->Gw.ensure(nw * ncol);
  tau_to_w_ff(c, Sig, c->Sw.p, ncol);
  tau_to_w_ff(c, G, c->Gw.p, ncol);
  const auto e_w = k_traces(c, c->Sw.p, c->Gw.p, nw, 0);
  std::complex<double> e = 0;
  for (int64_t t = 0; t < c->nt; ++t) {
    std::complex<double> et = 0;
    for (int64_t w = 0; w < nw; ++w) {
      const double2 T = c->Ttw_ff_h[t * nw + w];
      et += std::complex<double>(T.x, T.y) * e_w[w];
    }
    e += std::complex<double>(c->T_beta[t].x, c->T_beta[t].y) * et;
  }
  return (-0.5 * 2.0 * e).real();  // spin factor 2 for ns = 1
}

// e_1e = 2 sum_k w_k Tr[Dm H0], e_hf = 2 sum_k w_k Tr[Dm F] / 2 (scf_common.cpp:44-77)
void hf_energy_device(Ctx* c, double* e_1e, double* e_hf) {
  *e_1e = 2.0 * k_traces(c, c->Dm.p, c->H0.p, 1, 0)[0].real();
  *e_hf = 2.0 * 0.5 * k_traces(c, c->Dm.p, c->F.p, 1, 0)[0].real();
}

// Commutator residual (vspace_fock_sigma.hpp commutator_t) of (F, Sigma) with G_in:
// out(tau) = w_to_tau[G(iw) X(iw) - X(iw) G(iw)], X = (iw + mu) S - H0 - F - Sigma(iw).
void commutator_device(Ctx* c, const double2* F, const double2* Sig, const double2* Gin,
                       double2* out) {
  const int64_t nk = c->nk, nb = c->nb, ncol = nk * nb * nb, nw = c->nwf;
  c->Sw.ensure(nw * ncol);
  c->Gw.ensure(nw * ncol);
  c->Xw.ensure(nw * ncol);
  tau_to_w_ff(c, Gin, c->Gw.p, ncol);
  tau_to_w_ff(c, Sig, c->Sw.p, ncol);
  cq::build_dyson_matrix(c->Sov.p, c->H0.p, F, c->Sw.p, c->Xw.p, c->dwnf.p, c->beta, c->mu, nw, nk,
                         nb, c->st);
  // C = G X, then C -= X G (C in the Sigma(iw) buffer)
  zgemm_rm(c, 'N', 'N', nb, nb, nb, make_double2(1, 0), c->Gw.p, nb, nb * nb, c->Xw.p, nb, nb * nb,
           make_double2(0, 0), c->Sw.p, nb, nb * nb, nw * nk);
  zgemm_rm(c, 'N', 'N', nb, nb, nb, make_double2(-1, 0), c->Xw.p, nb, nb * nb, c->Gw.p, nb, nb * nb,
           make_double2(1, 0), c->Sw.p, nb, nb * nb, nw * nk);
  w_to_tau_ff(c, c->Sw.p, out, ncol);
}

// diag Sigma_ii^k(i w_n) of Sig(tau) into out (nwf, nk * nb)
void sigma_diag_w(Ctx* c, const double2* Sig, double2* out) {
  const int64_t nkb = c->nk * c->nb;
  c->dtmp.ensure(std::max(c->nt, c->nwf) * nkb);
  cq::extract_diag(Sig, c->dtmp.p, c->nb, c->nt * c->nk, c->st);
  zgemm_rm(c, 'N', 'N', c->nwf, nkb, c->nt, make_double2(1, 0), c->dTwt_ff.p, c->nt, 0, c->dtmp.p,
           nkb, 0, make_double2(0, 0), out, nkb, 0, 1);
}

// Sig(tau) += Ttw_ff diag(delta(i w)), then Hermitian again
void add_diag_w(Ctx* c, const double2* delta_w, double2* Sig) {
  const int64_t nkb = c->nk * c->nb;
  c->dtmp.ensure(std::max(c->nt, c->nwf) * nkb);
  zgemm_rm(c, 'N', 'N', c->nt, nkb, c->nwf, make_double2(1, 0), c->dTtw_ff.p, c->nwf, 0, delta_w,
           nkb, 0, make_double2(0, 0), c->dtmp.p, nkb, 0, 1);
  cq::add_diag(Sig, c->dtmp.p, c->nb, c->nt * c->nk, c->st);
  cq::hermitize_c128(Sig, c->nb, c->nt * c->nk, c->st);
}

// append diag Sigma_in(i w) to the four-iterate history (oldest dropped)
void push_history(Ctx* c, const double2* Sig) {
  const int64_t nel = c->nwf * c->nk * c->nb;
  c->dhist.ensure(5 * nel);
  if (c->nhist == 4) {
    CQ_CHECK_CUDA(cudaMemcpyAsync(c->dhist.p, c->dhist.p + nel, 3 * nel * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, c->st));
    c->nhist = 3;
  }
  sigma_diag_w(c, Sig, c->dhist.p + c->nhist * nel);
  ++c->nhist;
}

// Commutator DIIS step (diis_t::solve, diis_t.hpp:58-100) on the device vectors.  FS holds
// (F, Sigma) contiguous; returns (conv_F, conv_Sigma) and overwrites FS with the new state.
std::pair<double, double> diis_device(Ctx* c, double2* FS, int64_t it) {
  const int64_t nF = c->nk * c->nb * c->nb, nS = c->nt * nF, nFS = nF + nS;
  auto new_vec = [&](int64_t n) {
    auto b = std::make_unique<DevBuf<double2>>();
    b->ensure(n);
    return b;
  };
  auto copy = [&](double2* dst, const double2* src, int64_t n) {
    CQ_CHECK_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
  };
  auto damping = [&]() {
    const double m = c->mixing;
    cq::axpby_c128(c->prevFS.p, FS, 1.0 - m, m, nFS, c->st);
    return std::make_pair(cq::maxabs_diff(c->prevFS.p, FS, nF, c->red, c->st),
                          cq::maxabs_diff(c->prevFS.p + nF, FS + nF, nS, c->red, c->st));
  };
  // add (x = FS, residual of FS) to the subspaces, dropping the oldest pair when full
  auto add_residual = [&]() {
    if ((int64_t)c->dr.size() >= c->max_subsp) {
      c->dr.erase(c->dr.begin());
      c->dx.erase(c->dx.begin());
      const int64_t n = (int64_t)std::llround(std::sqrt((double)c->dB.size()));
      std::vector<std::complex<double>> B((n - 1) * (n - 1));
      for (int64_t i = 1; i < n; ++i)
        for (int64_t j = 1; j < n; ++j) B[(i - 1) * (n - 1) + (j - 1)] = c->dB[i * n + j];
      c->dB = B;
    }
    auto r = new_vec(nS);
    commutator_device(c, FS, FS + nF, c->Gin.p, r->p);
    const int64_t n = (int64_t)c->dr.size();
    std::vector<std::complex<double>> B((n + 1) * (n + 1));
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = 0; j < n; ++j) B[i * (n + 1) + j] = c->dB[i * n + j];
    for (int64_t i = 0; i < n; ++i) {
      const std::complex<double> o = cq::dotc(c->dr[i]->p, r->p, nS, c->red, c->st);
      B[i * (n + 1) + n] = o;
      B[n * (n + 1) + i] = std::conj(o);
    }
    B[n * (n + 1) + n] = cq::dotc(r->p, r->p, nS, c->red, c->st);
    c->dB = B;
    c->dr.push_back(std::move(r));
    auto x = new_vec(nFS);
    copy(x->p, FS, nFS);
    c->dx.push_back(std::move(x));
  };
  if ((int64_t)c->dx.size() == 1 || it < c->diis_start) {
    if (c->dx.size() <= 1) {
      auto x = new_vec(nFS);
      copy(x->p, FS, nFS);
      c->dx.push_back(std::move(x));
    } else {
      add_residual();
    }
    return damping();
  }
  add_residual();
  const int64_t n = (int64_t)c->dr.size();
  if (n <= 1) return damping();
  // compute_coefs_c1 (diis_alg.hpp:330-370): pseudo-inverse of Re B on its eigenbasis
  std::vector<double> B(n * n);
  for (int64_t i = 0; i < n * n; ++i) B[i] = c->dB[i].real();
  std::vector<double> ev, U;
  cq::sym_eigen(B, n, ev, U);
  const double emax = *std::max_element(ev.begin(), ev.end());
  const double emin = *std::min_element(ev.begin(), ev.end());
  const double cond = emax / emin;
  std::vector<double> xcoef(n, 0.0);
  for (int64_t k = 0; k < n; ++k) {
    if (!(ev[k] * cond > 1e-12)) continue;
    double proj = 0;  // u_k . 1
    for (int64_t i = 0; i < n; ++i) proj += U[i * n + k];
    for (int64_t i = 0; i < n; ++i) xcoef[i] += U[i * n + k] * proj / ev[k];
  }
  double sum = 0;
  for (double v : xcoef) sum += v;
  // make_linear_comb (vspace.h): coefficients aligned with the newest x-vectors
  c->Sw.ensure(std::max<int64_t>(nFS, c->nwf * nF));
  double2* R = c->Sw.p;
  CQ_CHECK_CUDA(cudaMemsetAsync(R, 0, nFS * sizeof(double2), c->st));
  const int64_t nx = (int64_t)c->dx.size();
  for (int64_t i = 0; i < std::min(nx, n); ++i)
    cq::axpy_c128(c->dx[nx - 1 - i]->p, R, make_double2(xcoef[n - 1 - i] / sum, 0.0), nFS, c->st);
  const double cF = cq::maxabs_diff(FS, R, nF, c->red, c->st);
  const double cS = cq::maxabs_diff(FS + nF, R + nF, nS, c->red, c->st);
  copy(FS, R, nFS);
  return {cF, cS};
}

// the symmetry-reduced (IBZ) k-space path and coqui_b200_set_symmetry
#include "ctx_sym.cuh"

// =======================================================================================
// ABI
// =======================================================================================
extern "C" {

const char* coqui_b200_version(void) { return kVersion; }

int coqui_b200_create(coqui_b200_ctx** out, const coqui_b200_dims* dims) {
  if (!out || !dims) return COQUI_B200_EINVAL;
  *out = nullptr;
  std::unique_ptr<Ctx> c(new (std::nothrow) Ctx());
  if (!c) return COQUI_B200_ENOMEM;
  const coqui_b200_dims& d = *dims;
  if (d.ns != 1 || d.nk < 1 || d.nb < 1 || d.Np < 1 || d.nt_f < 2 || d.nw_b < 1 ||
      d.kp_grid[0] * d.kp_grid[1] * d.kp_grid[2] != d.nk ||
      (d.precision_mode != COQUI_B200_FP64 && d.precision_mode != COQUI_B200_MIXED))
    return COQUI_B200_EINVAL;
  c->d = d;
  c->dev = d.device;
  int rc = guarded(c.get(), [&] {
    c->ns = d.ns;
    c->nk = c->nq = d.nk;
    c->nb = d.nb;
    c->Np = d.Np;
    c->nt = d.nt_f;
    c->nth = (d.nt_f + 1) / 2;
    c->nwb = d.nw_b;
    c->nwh = (d.nw_b + 1) / 2;
    c->nmax = std::max(c->nth, c->nwh);
    c->g = KGrid{(int)d.kp_grid[0], (int)d.kp_grid[1], (int)d.kp_grid[2]};
    CQ_REQUIRE(c->g.n0 <= 8 && c->g.n1 <= 8 && c->g.n2 <= 8, COQUI_B200_EUNSUPPORTED,
               "k-grid edges above 8 are not supported");
    c->mode = d.precision_mode;
    CQ_CHECK_CUDA(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    CQ_CHECK_CUDA(cudaStreamCreateWithFlags(&c->cs, cudaStreamNonBlocking));
    CQ_CHECK_CUDA(cudaEventCreateWithFlags(&c->ev_st, cudaEventDisableTiming));
    c->prof.st = c->st;
    cq::upload_twiddles();
    c->launch_base = cq::launches_total();
  });
  if (rc != COQUI_B200_OK) {
    coqui_b200_destroy(c.release());
    return rc;
  }
  *out = c.release();
  return COQUI_B200_OK;
}

void coqui_b200_destroy(coqui_b200_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->cs) cudaStreamSynchronize(c->cs);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->rexec) cudaGraphExecDestroy(c->rexec);
  for (auto* b : {&c->X, &c->V, &c->L, &c->LH, &c->chi, &c->G, &c->Sig, &c->Tproj, &c->stage,
                  &c->dTwt, &c->dTtw, &c->eps, &c->Gx})
    b->release();
  c->Gcache.release();
  for (cudaEvent_t e : c->up_ev) cudaEventDestroy(e);
  if (c->ev_st) cudaEventDestroy(c->ev_st);
  if (c->cs) cudaStreamDestroy(c->cs);
  c->fac.release();
  c->dTwtR.release();
  c->dTtwR.release();
  c->Gp.release();
  c->Gn.release();
  c->PW.release();
  c->dyn.release();
  c->Lc.release();
  c->LHc.release();
  c->Xtc.release();
  for (auto& m : c->marks) cudaEventDestroy(m.second);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

const char* coqui_b200_last_error(const coqui_b200_ctx* c) {
  return c ? c->err.c_str() : "null context";
}

int64_t coqui_b200_kernel_launches(const coqui_b200_ctx* c) {
  return c ? cq::launches_total() - c->launch_base : 0;
}

int coqui_b200_last_timings(const coqui_b200_ctx* c, char* names, int name_len, double* ms, int n) {
  if (!c) return COQUI_B200_EINVAL;
  int k = 0;
  for (const auto& p : c->last_ms) {
    if (k >= n) break;
    if (names && name_len > 0) {
      std::strncpy(names + (size_t)k * name_len, p.first.c_str(), name_len - 1);
      names[(size_t)k * name_len + name_len - 1] = 0;
    }
    if (ms) ms[k] = p.second;
    ++k;
  }
  return k;
}

int coqui_b200_set_ir(coqui_b200_ctx* c, const double* Twt_bb, const double* Ttw_bb,
                      const double* T_beta_t_ff, const double* tau_mesh_x) {
  return guarded(c, [&] {
    CQ_REQUIRE(Twt_bb && Ttw_bb && T_beta_t_ff && tau_mesh_x, COQUI_B200_EINVAL, "null IR table");
    const int64_t nt = c->nt, nwb = c->nwb, nth = c->nth, nwh = c->nwh;
    // thc_gw.cpp:56-66 particle-hole symmetry of the tau mesh
    for (int64_t it = 0; it < nt; ++it) {
      const double diff = std::abs(tau_mesh_x[it]) - std::abs(tau_mesh_x[nt - it - 1]);
      CQ_REQUIRE(diff <= 1e-6, COQUI_B200_EPHSYM,
                 "IAFT grid is not compatible with particle-hole symmetry");
    }
    auto at = [](const double* p, int64_t i) { return make_double2(p[2 * i], p[2 * i + 1]); };
    (void)nth;
    (void)nwh;
    cq::ph_symmetric_matrices(Twt_bb, Ttw_bb, nt, nwb, c->Twt_pos, c->Ttw_pos);
    c->Ttw_bb.resize(nt * nwb);
    for (int64_t i = 0; i < nt * nwb; ++i) c->Ttw_bb[i] = at(Ttw_bb, i);
    c->T_beta.resize(nt);
    for (int64_t i = 0; i < nt; ++i) c->T_beta[i] = at(T_beta_t_ff, i);
    c->dTwt.ensure(c->Twt_pos.size());
    c->dTtw.ensure(c->Ttw_pos.size());
    upload(c, c->dTwt.p, c->Twt_pos.data(), c->Twt_pos.size() * sizeof(double2));
    upload(c, c->dTtw.p, c->Ttw_pos.data(), c->Ttw_pos.size() * sizeof(double2));
    // The particle-hole symmetric matrices are real up to rounding (|Im| ~ 1e-15 |Re|);
    // then the transform runs with the real parts only.
    double re_max = 0, im_max = 0;
    for (const auto* v : {&c->Twt_pos, &c->Ttw_pos})
      for (const double2& z : *v) {
        re_max = std::max(re_max, std::abs(z.x));
        im_max = std::max(im_max, std::abs(z.y));
      }
    c->ir_real = im_max <= 1e-12 * re_max;
    if (c->ir_real) {
      std::vector<double> a(c->Twt_pos.size()), b(c->Ttw_pos.size());
      for (size_t i = 0; i < a.size(); ++i) a[i] = c->Twt_pos[i].x;
      for (size_t i = 0; i < b.size(); ++i) b[i] = c->Ttw_pos[i].x;
      c->dTwtR.ensure(a.size());
      c->dTtwR.ensure(b.size());
      upload(c, c->dTwtR.p, a.data(), a.size() * sizeof(double));
      upload(c, c->dTtwR.p, b.data(), b.size() * sizeof(double));
      CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    }
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->have_ir = true;
    c->gcache_valid = false;
  });
}

int coqui_b200_set_kmesh(coqui_b200_ctx* c, const double* kpts, const double* lattv,
                         const double* chi_bar_qP) {
  return guarded(c, [&] {
    CQ_REQUIRE(kpts && lattv, COQUI_B200_EINVAL, "null k-mesh");
    const int64_t nk = c->nk;
    const int n[3] = {c->g.n0, c->g.n1, c->g.n2};
    // The device DFT equals the reference's dense f_Rk / f_kR (kpoint_utils.hpp:461-705)
    // when k_i = (i0 b0/n0 + i1 b1/n1 + i2 b2/n2) in lexicographic order, b = 2 pi lattv^-T.
    for (int64_t k = 0; k < nk; ++k) {
      const int64_t idx[3] = {k / (n[1] * n[2]), (k / n[2]) % n[1], k % n[2]};
      for (int j = 0; j < 3; ++j) {
        // fractional coordinate along lattice vector j: k . a_j / (2 pi)
        double f = 0;
        for (int x = 0; x < 3; ++x) f += kpts[k * 3 + x] * lattv[j * 3 + x];
        f /= 2.0 * 3.14159265358979323846;
        const double want = (double)idx[j] / n[j];
        const double dlt = f - want;
        CQ_REQUIRE(std::abs(dlt - std::round(dlt)) < 1e-8, COQUI_B200_EUNSUPPORTED,
                   "k-points are not a Gamma-centred grid in lexicographic order");
      }
    }
    // dielectric-head prefactors (g0_div_utils.hpp:196-207) and the q of the reported head:
    // the first smallest nonzero |q| (find_smallest_qabs, g0_div_utils.hpp:263-282; q = 0
    // itself has a vanishing prefactor), q = 0 for a single q-point
    const double* a = lattv;
    const double vol = std::abs(a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                                a[2] * (a[3] * a[7] - a[4] * a[6]));
    const double fpi = 4.0 * 3.14159265358979323846;
    c->head_fac.resize(nk);
    double best = -1;
    c->q_smallest = 0;
    c->qnorm.resize(nk);
    c->qz.resize(nk);
    for (int64_t q = 0; q < nk; ++q) {
      const double q2 = kpts[3 * q] * kpts[3 * q] + kpts[3 * q + 1] * kpts[3 * q + 1] +
                        kpts[3 * q + 2] * kpts[3 * q + 2];
      c->head_fac[q] = q2 / fpi * vol;
      const double norm = std::sqrt(q2);
      c->qnorm[q] = norm;
      c->qz[q] = kpts[3 * q + 2];
      if (nk > 1 && norm > 0.0 && (best < 0 || norm < best)) {
        best = norm;
        c->q_smallest = q;
      }
    }
    c->fac.ensure(nk);
    upload(c, c->fac.p, c->head_fac.data(), nk * sizeof(double));
    c->chi.ensure((size_t)nk * c->Np);
    if (chi_bar_qP)
      upload(c, c->chi.p, chi_bar_qP, (size_t)nk * c->Np * sizeof(double2));
    else
      CQ_CHECK_CUDA(cudaMemsetAsync(c->chi.p, 0, (size_t)nk * c->Np * sizeof(double2), c->st));
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->have_k = true;
    c->gcache_valid = false;
    c->vr_valid = false;
    c->eps_raw_valid = false;
  });
}

int coqui_b200_set_thc(coqui_b200_ctx* c, const double* X_skPa, const double* V_qPQ) {
  return guarded(c, [&] {
    CQ_REQUIRE(X_skPa && V_qPQ, COQUI_B200_EINVAL, "null THC data");
    const int64_t nk = c->nk, Np = c->Np, nb = c->nb;
    c->X.ensure((size_t)nk * Np * nb);
    c->V.ensure((size_t)nk * Np * Np);
    upload(c, c->X.p, X_skPa, (size_t)nk * Np * nb * sizeof(double2));
    upload(c, c->V.p, V_qPQ, (size_t)nk * Np * Np * sizeof(double2));
    // NaN or Inf would pass the factorisation's pivot test (it compares with zero): refuse them
    c->flag.ensure(1);
    CQ_CHECK_CUDA(cudaMemsetAsync(c->flag.p, 0, sizeof(int), c->st));
    cq::launch_check_finite(c->X.p, nk * Np * nb, c->flag.p, c->st);
    cq::launch_check_finite(c->V.p, nk * Np * Np, c->flag.p, c->st);
    int bad = 0;
    CQ_CHECK_CUDA(cudaMemcpyAsync(&bad, c->flag.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    CQ_REQUIRE(!bad, COQUI_B200_EINVAL, "X or V holds NaN or Inf values");
    // V^q = L L^H once per q (FP64)
    c->L.ensure((size_t)nk * Np * Np);
    c->LH.ensure((size_t)nk * Np * Np);
    CQ_CHECK_CUDA(cudaMemcpyAsync(c->L.p, c->V.p, (size_t)nk * Np * Np * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, c->st));
    int info = cq::cholesky_lower_batched(c->L.p, Np, nk, c->st);
    CQ_REQUIRE(info == 0, COQUI_B200_ENOTHPD, "Coulomb matrix V^q is not positive definite");
    cq::launch_zero_upper_and_adjoint(c->L.p, c->LH.p, Np, nk, c->st);
    if (c->mode == COQUI_B200_MIXED) {
      cq::tc_pack_X(c->Xtc, c->X.p, nk, Np, nb, c->st);
      c->Lc.ensure((size_t)nk * Np * Np);
      c->LHc.ensure((size_t)nk * Np * Np);
      cq::to_c64(c->L.p, c->Lc.p, Np, Np, nk, false, c->st);
      cq::to_c64(c->LH.p, c->LHc.p, Np, Np, nk, false, c->st);
    }
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->have_thc = true;
    if (c->sym) {
      c->sym->thc_ready = false;
      c->sym->w_valid = false;
    }
    c->gcache_valid = false;
    c->w_valid = false;
    c->vr_valid = false;
    c->tdiv_valid = false;
    c->eps_raw_valid = false;
  });
}

int coqui_b200_primary_to_aux(coqui_b200_ctx* c, int64_t n_tau, const double* O_tskab,
                              double* O_tskPQ) {
  return guarded(c, [&] {
    require_ready(c, true, false, false);
    CQ_REQUIRE(n_tau >= 1 && O_tskab && O_tskPQ, COQUI_B200_EINVAL, "bad arguments");
    const int64_t nk = c->nk, nb = c->nb, Np = c->Np, ncol = Np * Np;
    const size_t gsz = (size_t)nk * nb * nb;
    c->Gx.ensure(gsz);  // not c->G: a resident G stays valid
    c->Gp.ensure((size_t)nk * ncol * c->elem());
    c->stage.ensure((size_t)nk * ncol);
    for (int64_t t = 0; t < n_tau; ++t) {
      upload(c, c->Gx.p, O_tskab + 2 * t * gsz, gsz * sizeof(double2));
      project_p2a(c, c->Gx.p, c->Gp.p);
      const double2* src = (const double2*)c->Gp.p;
      if (c->mode == COQUI_B200_MIXED) {
        cq::launch_to_c128<float>((float2*)c->Gp.p, c->stage.p, nk * ncol, c->st);
        src = c->stage.p;
      }
      download(c, O_tskPQ + 2 * t * nk * ncol, src, (size_t)nk * ncol * sizeof(double2));
      CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    }
  });
}

int coqui_b200_aux_to_primary(coqui_b200_ctx* c, int64_t n_tau, const double* O_tskPQ,
                              double* O_tskab) {
  return guarded(c, [&] {
    require_ready(c, true, false, false);
    CQ_REQUIRE(n_tau >= 1 && O_tskab && O_tskPQ, COQUI_B200_EINVAL, "bad arguments");
    const int64_t nk = c->nk, nb = c->nb, Np = c->Np, ncol = Np * Np;
    const size_t gsz = (size_t)nk * nb * nb;
    c->Sig.ensure(gsz);
    c->Gp.ensure((size_t)nk * ncol * c->elem());
    c->stage.ensure((size_t)nk * ncol);
    for (int64_t t = 0; t < n_tau; ++t) {
      if (c->mode == COQUI_B200_FP64) {
        upload(c, c->Gp.p, O_tskPQ + 2 * t * nk * ncol, (size_t)nk * ncol * sizeof(double2));
      } else {
        upload(c, c->stage.p, O_tskPQ + 2 * t * nk * ncol, (size_t)nk * ncol * sizeof(double2));
        cq::launch_from_c128<float>(c->stage.p, (float2*)c->Gp.p, nk * ncol, c->st);
      }
      project_a2p(c, c->Gp.p, c->Sig.p);
      download(c, O_tskab + 2 * t * gsz, c->Sig.p, gsz * sizeof(double2));
      CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    }
  });
}

int coqui_b200_eval_pi(coqui_b200_ctx* c, const double* G_tskij, double* Pi_tqPQ) {
  return guarded(c, [&] {
    require_ready(c, true, true, true);
    if (c->sym) {
      sym_eval_pi(c, G_tskij, Pi_tqPQ);
      return;
    }
    c->begin_timing();
    upload_G(c, G_tskij);
    c->mark("h2d_G");
    eval_pi_device(c);
    c->mark("EVALUATE_PI_R");
    if (Pi_tqPQ) {
      const int64_t n = c->nth * c->nq * c->Np * c->Np;
      if (c->mode == COQUI_B200_FP64) {
        download(c, Pi_tqPQ, c->PW.p, n * sizeof(double2));
      } else {
        // stream out in slabs of one tau through the staging buffer
        const int64_t slab = c->nq * c->Np * c->Np;
        c->stage.ensure(slab);
        for (int64_t t = 0; t < c->nth; ++t) {
          cq::launch_to_c128<float>((float2*)c->PW.p + t * slab, c->stage.p, slab, c->st);
          download(c, Pi_tqPQ + 2 * t * slab, c->stage.p, slab * sizeof(double2));
        }
      }
    }
    c->mark("d2h");
    c->end_timing();
  });
}

namespace {

// Pi(iW) in the PW buffer -> W(iW) (want_w) and/or per-problem log det / trace (want_e).
void dyson_all(Ctx* c, bool want_w, bool want_e, std::vector<double>* logdet,
               std::vector<double2>* tr) {
  cq::DysonArgs a;
  a.Np = c->Np;
  a.nq = c->nq;
  a.nw = c->nwh;
  a.L = c->L.p;
  a.LH = c->LH.p;
  a.V = c->V.p;
  a.Lc = c->Lc.p;
  a.LHc = c->LHc.p;
  a.want_w = want_w;
  a.want_e = want_e;
  a.mixed = (c->mode == COQUI_B200_MIXED);
  a.PW = c->PW.p;
  a.prof = &c->prof;
  const int64_t nprob = c->nwh * c->nq;
  c->dinfo.ensure(nprob);
  c->dlogdet.ensure(nprob);
  c->dtrace.ensure(nprob);
  a.info = c->dinfo.p;
  a.logdet = c->dlogdet.p;
  a.trace = c->dtrace.p;
  a.defer_check = c->capturing || c->defer_dyson_check;
  a.keep_scratch = c->capturing;
  std::vector<double> ld;
  std::vector<double2> t;
  cq::dyson_run(a, c->dyn, c->st, want_e ? &ld : nullptr, want_e ? &t : nullptr);
  if (logdet) *logdet = std::move(ld);
  if (tr) *tr = std::move(t);
}

void update_w_device(Ctx* c) {
  eval_pi_device(c);
  c->mark("EVALUATE_PI_R");
  ir_inplace(c, (int)c->nth, (int)c->nwh, c->dTwt.p);
  c->mark("IMAG_FT_TtoW");
  dyson_all(c, true, false, nullptr, nullptr);
  c->mark("EVALUATE_W");
  ir_inplace(c, (int)c->nwh, (int)c->nth, c->dTtw.p);
  c->mark("IMAG_FT_WtoT");
  c->w_valid = true;
  c->w_in_R = false;
  c->eps_raw_valid = false;
}

// the treatment in effect: with one q-point every treatment is ignore_g0
// (g0_div_utils.hpp:68-72, thc_gw.icc:454-458)
bool div_active(const Ctx* c) { return c->div != 0 && c->nq > 1; }

// eps^-1 head per (tau, q) of the current W, which must be in q-space (eval_eps_inv_q,
// g0_div_utils.hpp:180-214) -> c->eps_raw (nth, nq)
void eps_raw_heads(Ctx* c) {
  cq::Prof::Scope sc(&c->prof, "eps_head");
  CQ_REQUIRE(!c->w_in_R, COQUI_B200_EINVAL, "eps head: W is not in q-space");
  c->eps.ensure((size_t)c->nth * c->nq);
  if (c->mode == COQUI_B200_FP64)
    cq::launch_eps_head<double>((double2*)c->PW.p, c->chi.p, c->fac.p, c->eps.p, c->nth, c->nq,
                                c->Np, c->st);
  else
    cq::launch_eps_head<float>((float2*)c->PW.p, c->chi.p, c->fac.p, c->eps.p, c->nth, c->nq,
                               c->Np, c->st);
  c->eps_raw.resize((size_t)c->nth * c->nq);
  download(c, c->eps_raw.data(), c->eps.p, c->eps_raw.size() * sizeof(double2));
  CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
  c->eps_raw_valid = true;
}

// eps_inv_head_t (g0_div_utils.hpp:55-111): c->head_h (nth) from eps (nth, nq) over the
// q-points with norms qnorm and z components qz.  ignore_g0 and gygi: the first smallest
// nonzero |q| (q_smallest).  gygi_extrplt(_2d): through the q with 0 < |q| <= 0.8 (q_z = 0 for
// _2d; distinct |q| only, filter_qpts :26-42), per bosonic frequency (tau_to_w_PHsym), the
// least-squares quadratic in |q| extrapolated to q = 0 (extrapolate_to_q0 :284-311), back with
// w_to_tau_PHsym; the first such q alone when fewer than 3.
void select_head_from(Ctx* c, const std::vector<double2>& eps, int64_t nq,
                      const std::vector<double>& qnorm, const std::vector<double>& qz,
                      int64_t q_smallest) {
  const int64_t nth = c->nth, nwh = c->nwh;
  c->head_h.assign(nth, make_double2(0, 0));
  const int div = nq == 1 ? 0 : c->div;
  int64_t col = q_smallest;
  if (div >= 2) {
    std::vector<int64_t> idx;
    std::set<double> seen;
    for (int64_t q = 0; q < nq; ++q) {
      const double n = qnorm[q];
      if (n > 0.0 && n <= 0.8 && (div != 3 || qz[q] == 0.0) && seen.insert(n).second)
        idx.push_back(q);
    }
    CQ_REQUIRE(!idx.empty(), COQUI_B200_EINVAL,
               "gygi_extrplt: no q-point with 0 < |q| <= 0.8 for the extrapolation");
    if (idx.size() >= 3) {
      using cd = std::complex<double>;
      const size_t m = idx.size();
      // normal equations of A(i, j) = |q_i|^j, j = 0..2
      double a[3][3] = {};
      for (size_t i = 0; i < m; ++i) {
        const double Q = qnorm[idx[i]], p[3] = {1.0, Q, Q * Q};
        for (int j = 0; j < 3; ++j)
          for (int l = 0; l < 3; ++l) a[j][l] += p[j] * p[l];
      }
      // first row of (A^T A)^{-1} (cofactors of the symmetric 3 x 3)
      const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
      const double c01 = a[0][2] * a[2][1] - a[0][1] * a[2][2];
      const double c02 = a[0][1] * a[1][2] - a[0][2] * a[1][1];
      const double det = a[0][0] * c00 + a[1][0] * c01 + a[2][0] * c02;
      CQ_REQUIRE(det != 0.0, COQUI_B200_EINVAL, "gygi_extrplt: singular fit");
      const double r0[3] = {c00 / det, c01 / det, c02 / det};
      std::vector<cd> e0(nwh);
      for (int64_t n = 0; n < nwh; ++n) {
        cd atb[3] = {};
        for (size_t i = 0; i < m; ++i) {
          cd ew = 0;
          for (int64_t t = 0; t < nth; ++t) {
            const double2 T = c->Twt_pos[n * nth + t], e = eps[t * nq + idx[i]];
            ew += cd(T.x, T.y) * cd(e.x, e.y);
          }
          const double Q = qnorm[idx[i]], p[3] = {1.0, Q, Q * Q};
          for (int j = 0; j < 3; ++j) atb[j] += p[j] * ew;
        }
        e0[n] = r0[0] * atb[0] + r0[1] * atb[1] + r0[2] * atb[2];
      }
      for (int64_t t = 0; t < nth; ++t) {
        cd h = 0;
        for (int64_t n = 0; n < nwh; ++n) {
          const double2 T = c->Ttw_pos[t * nwh + n];
          h += cd(T.x, T.y) * e0[n];
        }
        c->head_h[t] = make_double2(h.real(), h.imag());
      }
      return;
    }
    col = idx[0];
  }
  for (int64_t t = 0; t < nth; ++t) c->head_h[t] = eps[t * nq + col];
}
void select_head(Ctx* c) {
  select_head_from(c, c->eps_raw, c->nq, c->qnorm, c->qz, c->q_smallest);
}

// the eps^-1 head of the current W (nth complex values as (re, im) into out, if not null)
void eps_head(Ctx* c, double* out) {
  if (!c->eps_raw_valid) eps_raw_heads(c);
  select_head(c);
  if (out)
    for (int64_t t = 0; t < c->nth; ++t) {
      out[2 * t] = c->head_h[t].x;
      out[2 * t + 1] = c->head_h[t].y;
    }
}

// gw_t::Sigma_div_correction (thc_gw.icc:446-526) on a device Sigma (FP64), for the gygi
// treatments: Sigma(t, k) += -madelung Re head(t_pos) T^k G(t, k) T^kH with
// T^k = X^kH diag(conj chi_head) X^k, t_pos = t below nt_half, else nt - 1 - t; nk k-points
// with collocation X (nk, Np, nb), G and Sigma (nt, nk, nb, nb); T^k kept in Tdiv while
// tdiv_valid.
void sigma_div_correction_on(Ctx* c, int64_t nk, const double2* X, const double2* G,
                             double2* Sig, DevBuf<double2>& Tdiv, bool& tdiv_valid) {
  cq::Prof::Scope sc(&c->prof, "sigma_div");
  const int64_t nb = c->nb, Np = c->Np, nt = c->nt, nth = c->nth, per = nb * nb;
  const int64_t nprob = nt * nk;
  if (!tdiv_valid) {
    Tdiv.ensure(nk * per);
    c->Tproj.ensure((size_t)nk * Np * nb);
    cq::scale_rows(X, c->chi0c.p, c->Tproj.p, nk, Np, nb, c->st);
    zgemm_rm(c, 'C', 'N', nb, nb, Np, make_double2(1, 0), X, nb, Np * nb, c->Tproj.p, nb,
             Np * nb, make_double2(0, 0), Tdiv.p, nb, per, nk);
    tdiv_valid = true;
  }
  std::vector<double> f(nt);
  for (int64_t t = 0; t < nt; ++t) f[t] = -c->madelung * c->head_h[t < nth ? t : nt - t - 1].x;
  c->divf.ensure(nt);
  upload(c, c->divf.p, f.data(), nt * sizeof(double));
  c->divY.ensure(nprob * per);
  // pointer arrays: (T, G, Y) for Y = T G, then (Y, T, Sigma) for Sigma += Y T^H
  c->divp_h.resize(6 * nprob);
  for (int64_t t = 0; t < nt; ++t)
    for (int64_t k = 0; k < nk; ++k) {
      const int64_t i = t * nk + k;
      c->divp_h[i] = Tdiv.p + k * per;
      c->divp_h[nprob + i] = G + i * per;
      c->divp_h[2 * nprob + i] = c->divY.p + i * per;
      c->divp_h[3 * nprob + i] = c->divY.p + i * per;
      c->divp_h[4 * nprob + i] = Tdiv.p + k * per;
      c->divp_h[5 * nprob + i] = Sig + i * per;
    }
  c->divp.ensure(6 * nprob);
  upload(c, c->divp.p, c->divp_h.data(), 6 * nprob * sizeof(const double2*));
  const double2* const* P = c->divp.p;
  zgemm_rm_ptrs(c, 'N', 'N', nb, nb, nb, make_double2(1, 0), P, nb, P + nprob, nb,
                make_double2(0, 0), const_cast<double2* const*>(P + 2 * nprob), nb, nprob);
  cq::scale_slices(c->divY.p, c->divf.p, nt, nk * per, c->st);
  zgemm_rm_ptrs(c, 'N', 'C', nb, nb, nb, make_double2(1, 0), P + 3 * nprob, nb, P + 4 * nprob,
                nb, make_double2(1, 0), const_cast<double2* const*>(P + 5 * nprob), nb, nprob);
}
void sigma_div_correction(Ctx* c) {
  sigma_div_correction_on(c, c->nk, c->X.p, c->G.p, c->Sig.p, c->Tdiv, c->tdiv_valid);
}

void download_w_qt(Ctx* c, double* dW_qtPQ) {
  const int64_t ncol = c->Np * c->Np;
  const int64_t per_q = c->nth * ncol;
  // one q at a time through the staging buffer (transposes (t, q) -> (q, t))
  c->stage.ensure(per_q);
  for (int64_t q = 0; q < c->nq; ++q) {
    if (c->mode == COQUI_B200_FP64)
      cq::launch_tq_to_qt_c128<double>((double2*)c->PW.p, c->stage.p, c->nth, c->nq, ncol, q, 1,
                                       c->st);
    else
      cq::launch_tq_to_qt_c128<float>((float2*)c->PW.p, c->stage.p, c->nth, c->nq, ncol, q, 1,
                                      c->st);
    download(c, dW_qtPQ + 2 * q * per_q, c->stage.p, per_q * sizeof(double2));
  }
}

// Sigma(tau) for all tau into c->Sig (device, complex128), thc_gw.icc:70-213 twice.
// host_out (may be null) receives Sigma_tskij; from page-locked memory it is filled chunk by
// chunk on the copy stream while the following chunks are computed.
void w_to_q_space(Ctx* c);

void sigma_device(Ctx* c, double* host_out) {
  CQ_REQUIRE(c->w_valid, COQUI_B200_EINVAL, "no screened interaction: call update_w or set_w");
  const int64_t nk = c->nk, nb = c->nb, Np = c->Np, ncol = Np * Np, nt = c->nt;
  const size_t slab = (size_t)nk * ncol * c->elem();
  const size_t gsz = (size_t)nk * nb * nb;
  c->Gp.ensure(slab);
  c->Gn.ensure(slab);
  c->Sig.ensure((size_t)nt * gsz);
  // the gygi treatments need the eps^-1 head of this W (thc_gw.icc:30-33): taken while W is
  // in q-space (a W left in R by an earlier call is transformed back once)
  const bool corr = div_active(c);
  if (corr) {
    CQ_REQUIRE(c->chi0c.n >= (size_t)Np, COQUI_B200_EINVAL,
               "the gygi treatments of Sigma need chi_head (coqui_b200_set_div_treatment)");
    if (!c->eps_raw_valid && c->w_in_R) w_to_q_space(c);
    eps_head(c, nullptr);
  }
  // W q -> R once (thc_gw.icc:148-153); stays in R until the next update
  if (!c->w_in_R) {
    cq::Prof::Scope sc(&c->prof, "dft_w");
    const double s = 1.0 / (double)nk;
    if (c->mode == COQUI_B200_FP64)
      cq::launch_dft_plain<double>((double2*)c->PW.p, ncol, c->g, -1, s, c->nth, c->nq * ncol,
                                   c->st);
    else
      cq::launch_dft_plain<float>((float2*)c->PW.p, ncol, c->g, -1, s, c->nth, c->nq * ncol,
                                  c->st);
    c->w_in_R = true;
  }
  c->mark("SIGMA_FT_W");
  // G_PQ(tau) of this G is still in the cache when the polarizability just ran: Sigma_PQ is
  // then formed in place there and projected back in batches
  unsigned char* cache = c->gcache_valid ? c->Gcache.p : nullptr;
  c->gcache_valid = false;
  // with the q -> 0 correction, Sigma leaves once it is complete
  const bool pipe_out = host_out && is_pinned(host_out) && !corr;
  for (int64_t i = 0; i < n_tau_chunks(c); ++i) {
    int64_t a, b;
    tau_chunk_range(c, i, &a, &b);
    const bool cached = cache && gchunk_cached(c, b);
    if (!cached) wait_G_chunk(c, i);
    for (int64_t it = a; it < b; ++it) {
      const bool minus = it < nt / 2;  // thc_gw.icc:59-61 writes Sigma(nt-1-it) for it < nt/2
      unsigned char* gp = c->Gp.p;
      unsigned char* gn = minus ? c->Gn.p : nullptr;
      if (cached) {
        gp = gslab(c, it);
        gn = minus ? gslab(c, nt - it - 1) : nullptr;
      } else {
        project_p2a(c, c->G.p + it * gsz, gp);
        if (minus) project_p2a(c, c->G.p + (nt - it - 1) * gsz, gn);
      }
      unsigned char* WR = c->PW.p + (size_t)it * c->nq * ncol * c->elem();
      {
        cq::Prof::Scope sc(&c->prof, "sigma_fused");
        if (c->mode == COQUI_B200_FP64)
          cq::launch_sigma_fused<double>((double2*)gp, (double2*)gn, (double2*)WR, (double2*)gp,
                                         (double2*)gn, ncol, c->g, c->st);
        else
          cq::launch_sigma_fused<float>((float2*)gp, (float2*)gn, (float2*)WR, (float2*)gp,
                                        (float2*)gn, ncol, c->g, c->st);
      }
      if (!cached) {
        project_a2p(c, gp, c->Sig.p + it * gsz);
        if (minus) project_a2p(c, gn, c->Sig.p + (nt - it - 1) * gsz);
      }
    }
    if (cached) {
      // for odd nt the middle slice is in both ranges (same values written twice)
      project_a2p(c, gslab(c, a), c->Sig.p + a * gsz, b - a);
      project_a2p(c, gslab(c, nt - b), c->Sig.p + (nt - b) * gsz, b - a);
    }
    if (pipe_out) {
      const size_t bytes = (size_t)(b - a) * gsz * sizeof(double2);
      double2* h = reinterpret_cast<double2*>(host_out);
      CQ_CHECK_CUDA(cudaEventRecord(c->ev_st, c->st));
      CQ_CHECK_CUDA(cudaStreamWaitEvent(c->cs, c->ev_st, 0));
      CQ_CHECK_CUDA(cudaMemcpyAsync(h + a * gsz, c->Sig.p + a * gsz, bytes, cudaMemcpyDeviceToHost, c->cs));
      CQ_CHECK_CUDA(cudaMemcpyAsync(h + (nt - b) * gsz, c->Sig.p + (nt - b) * gsz, bytes,
                                    cudaMemcpyDeviceToHost, c->cs));
    }
  }
  if (corr) sigma_div_correction(c);
  c->mark("EVALUATE_SIGMA_R");
  if (host_out) {
    if (pipe_out) {  // the compute stream's timeline ends when the last copy landed
      CQ_CHECK_CUDA(cudaEventRecord(c->ev_st, c->cs));
      CQ_CHECK_CUDA(cudaStreamWaitEvent(c->st, c->ev_st, 0));
    } else {
      download(c, host_out, c->Sig.p, (size_t)nt * gsz * sizeof(double2));
    }
    c->mark("d2h_Sigma");
  }
}

void w_to_q_space(Ctx* c) {
  if (!c->w_in_R) return;
  const int64_t ncol = c->Np * c->Np;
  if (c->mode == COQUI_B200_FP64)
    cq::launch_dft_plain<double>((double2*)c->PW.p, ncol, c->g, +1, 1.0, c->nth, c->nq * ncol,
                                 c->st);
  else
    cq::launch_dft_plain<float>((float2*)c->PW.p, ncol, c->g, +1, 1.0, c->nth, c->nq * ncol,
                                c->st);
  c->w_in_R = false;
}


// ---------------------------------------------------------------------------------------
// THC Hartree-Fock: hf_t::evaluate for q-independent THC without symmetry (thc_hf.cpp:21-60
// -> thc_hf.icc:17-272, npol = 1) and HF_K_correction (hf_t.cpp:45-84).
// ---------------------------------------------------------------------------------------

// V(R) = f_Rq V(q) (thc_hf.icc:143-152) in FP64, built once per set_thc
void ensure_v_R(Ctx* c) {
  if (c->vr_valid) return;
  const int64_t nk = c->nk, ncol = c->Np * c->Np;
  c->VR.ensure((size_t)nk * ncol);
  CQ_CHECK_CUDA(cudaMemcpyAsync(c->VR.p, c->V.p, (size_t)nk * ncol * sizeof(double2),
                                cudaMemcpyDeviceToDevice, c->st));
  cq::launch_dft_plain<double>(c->VR.p, ncol, c->g, -1, 1.0 / (double)nk, 1, nk * ncol, c->st);
  c->vr_valid = true;
}

// F (device, (nk, nb, nb)) <- J + K [- madelung S Dm S] of the density matrix Dm (device), in
// FP64 in both precision modes (one slice of the self-energy's work; F enters every G(i w)).
// K_PQ(R) = -D_PQ(R) V_PQ(R) takes the self-energy's route (projection, fused k -> R, product,
// R -> k, back-projection) with D(k) = X Dm X^H in place of G(tau) and V(R) in place of W(R).
// J: rho_Q = (2/nk) sum_k (X Dm X^H)_QQ (the R = 0 diagonal of thc_hf.icc:184-190),
// J = V(q=0) rho (:194-196), F += X^H diag(J) X.
void hf_device(Ctx* c, const double2* Dm, const double2* S, bool hartree, bool exchange, int div,
               double madelung, double2* F) {
  cq::Prof::Scope sc(&c->prof, "hf");
  const int64_t nk = c->nk, nb = c->nb, Np = c->Np, ncol = Np * Np;
  const int64_t nF = nk * nb * nb;
  if (exchange) {
    ensure_v_R(c);
    c->hfp.ensure((size_t)nk * ncol);
    p2a_fp64(c, Dm, c->hfp.p, 1);
    cq::launch_sigma_fused<double>(c->hfp.p, nullptr, c->VR.p, c->hfp.p, nullptr, ncol, c->g,
                                   c->st);
    a2p_fp64(c, c->hfp.p, F, 1);
  } else {
    CQ_CHECK_CUDA(cudaMemsetAsync(F, 0, nF * sizeof(double2), c->st));
  }
  if (hartree) {
    c->Tproj.ensure((size_t)nk * Np * nb);
    c->hfv.ensure(2 * Np);
    const double2 one = make_double2(1, 0), zero = make_double2(0, 0);
    zgemm_rm(c, 'N', 'N', Np, nb, nb, one, c->X.p, nb, Np * nb, Dm, nb, nb * nb, zero,
             c->Tproj.p, nb, Np * nb, nk);
    cq::aux_diag(c->Tproj.p, c->X.p, c->hfv.p, nk, Np, nb, 2.0 / (double)nk, c->st);
    zgemm_rm(c, 'N', 'N', Np, 1, Np, one, c->V.p, Np, 0, c->hfv.p, 1, 0, zero, c->hfv.p + Np, 1,
             0, 1);
    cq::scale_rows(c->X.p, c->hfv.p + Np, c->Tproj.p, nk, Np, nb, c->st);
    zgemm_rm(c, 'C', 'N', nb, nb, Np, one, c->X.p, nb, Np * nb, c->Tproj.p, nb, Np * nb, one, F,
             nb, nb * nb, nk);
  }
  if (exchange && div == 1) {
    c->hft.ensure(nF);
    zgemm_rm(c, 'N', 'N', nb, nb, nb, make_double2(1, 0), S, nb, nb * nb, Dm, nb, nb * nb,
             make_double2(0, 0), c->hft.p, nb, nb * nb, nk);
    zgemm_rm(c, 'N', 'N', nb, nb, nb, make_double2(-madelung, 0), c->hft.p, nb, nb * nb, S, nb,
             nb * nb, make_double2(1, 0), F, nb, nb * nb, nk);
  }
}

// One GW iteration of the resident G as a CUDA graph (update_w + Sigma, no host transfers).
// status of every (iW, q) factorisation of the last Dyson step, left on the device
void check_dyson_status(Ctx* c) {
  const int64_t nprob = c->nwh * c->nq;
  std::vector<int> info(nprob);
  CQ_CHECK_CUDA(cudaMemcpyAsync(info.data(), c->dinfo.p, nprob * sizeof(int), cudaMemcpyDeviceToHost,
                                c->st));
  CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
  for (int64_t i = 0; i < nprob; ++i)
    CQ_REQUIRE(info[i] == 0, COQUI_B200_ENOTHPD, "I - L^H Pi L is not positive definite");
}

// G_host / S_host: page-locked host buffers copied in / out inside the graph (chunked on the
// copy stream as in the directly launched path), or nullptr for the resident G and a Sigma
// left on the device.  The graph is replayed by the next call with the same buffers.
void gw_iteration_graph(Ctx* c, const double* G_host, double* S_host) {
  c->begin_timing();
  const bool replay = c->gexec && c->graph_call == c->calls - 1 && c->graph_g == G_host &&
                      c->graph_s == S_host;
  if (!replay) {
    if (c->gexec) {
      cudaGraphExecDestroy(c->gexec);
      c->gexec = nullptr;
    }
    c->g_pipelined = false;  // the resident G is complete on the device
    const int64_t l0 = cq::launches_total();
    CQ_CHECK_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed));
    c->capturing = true;
    cudaGraph_t g = nullptr;
    try {
      if (G_host) upload_G(c, G_host);
      update_w_device(c);
      sigma_device(c, S_host);
    } catch (...) {
      c->capturing = false;
      if (cudaStreamEndCapture(c->st, &g) == cudaSuccess && g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    c->capturing = false;
    CQ_CHECK_CUDA(cudaStreamEndCapture(c->st, &g));
    c->graph_launches = cq::launches_total() - l0;
    const cudaError_t e = cudaGraphInstantiate(&c->gexec, g, 0);
    cudaGraphDestroy(g);
    CQ_CHECK_CUDA(e);
    c->graph_g = G_host;
    c->graph_s = S_host;
  } else {
    cq::count_launch(c->graph_launches);  // the replay launches the captured kernels again
  }
  CQ_CHECK_CUDA(cudaGraphLaunch(c->gexec, c->st));
  c->mark("GW_ITERATION_GRAPH");
  c->graph_call = c->calls;
  check_dyson_status(c);  // factorisation status of every (iW, q) problem of this iteration
  c->end_timing();
}

// RPA energy of the resident G (or of a page-locked host G copied inside the graph) as one
// CUDA graph: polarizability, tau -> w, the factorisations with their log-determinants and
// traces left on the device; E_c is summed on the host from those afterwards.  Replayed by
// the next call with the same G argument.
void rpa_energy_graph(Ctx* c, const double* G_host, double* e_rpa) {
  c->begin_timing();
  const bool replay = c->rexec && c->rgraph_call == c->calls - 1 && c->rgraph_g == G_host;
  if (!replay) {
    if (c->rexec) {
      cudaGraphExecDestroy(c->rexec);
      c->rexec = nullptr;
    }
    c->g_pipelined = false;  // the resident G is complete on the device
    const int64_t l0 = cq::launches_total();
    CQ_CHECK_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed));
    c->capturing = true;
    cudaGraph_t g = nullptr;
    try {
      if (G_host) upload_G(c, G_host);
      eval_pi_device(c);
      ir_inplace(c, (int)c->nth, (int)c->nwh, c->dTwt.p);
      dyson_all(c, false, true, nullptr, nullptr);
    } catch (...) {
      c->capturing = false;
      if (cudaStreamEndCapture(c->st, &g) == cudaSuccess && g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    c->capturing = false;
    CQ_CHECK_CUDA(cudaStreamEndCapture(c->st, &g));
    c->rgraph_launches = cq::launches_total() - l0;
    const cudaError_t e = cudaGraphInstantiate(&c->rexec, g, 0);
    cudaGraphDestroy(g);
    CQ_CHECK_CUDA(e);
    c->rgraph_g = G_host;
  } else {
    cq::count_launch(c->rgraph_launches);
  }
  CQ_CHECK_CUDA(cudaGraphLaunch(c->rexec, c->st));
  c->mark("RPA_GRAPH");
  c->rgraph_call = c->calls;
  check_dyson_status(c);
  const int64_t nprob = c->nwh * c->nq;
  std::vector<double> ld(nprob);
  std::vector<double2> tr(nprob);
  CQ_CHECK_CUDA(cudaMemcpyAsync(ld.data(), c->dlogdet.p, nprob * sizeof(double),
                                cudaMemcpyDeviceToHost, c->st));
  CQ_CHECK_CUDA(cudaMemcpyAsync(tr.data(), c->dtrace.p, nprob * sizeof(double2),
                                cudaMemcpyDeviceToHost, c->st));
  CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
  for (double v : ld)
    CQ_REQUIRE(std::isfinite(v), COQUI_B200_ENOTHPD, "I - Pi V is not positive definite");
  *e_rpa = rpa_energy_from(c, ld, tr);
  c->end_timing();
}
}  // namespace

int coqui_b200_update_w(coqui_b200_ctx* c, const double* G_tskij, double* dW_qtPQ,
                        double* eps_inv_head) {
  return guarded(c, [&] {
    require_ready(c, true, true, true);
    if (c->sym) {
      c->begin_timing();
      sym_upload_g(c, G_tskij);
      c->mark("h2d_G");
      sym_update_w(c);
      if (eps_inv_head) {
        sym_eps_head(c, eps_inv_head);
        c->mark("EPS_INV_HEAD");
      }
      if (dW_qtPQ) {
        sym_download_w(c, dW_qtPQ);
        c->mark("d2h_W");
      }
      c->end_timing();
      return;
    }
    c->begin_timing();
    upload_G(c, G_tskij);
    c->mark("h2d_G");
    update_w_device(c);
    if (eps_inv_head) {
      eps_head(c, eps_inv_head);
      c->mark("EPS_INV_HEAD");
    }
    if (dW_qtPQ) {
      download_w_qt(c, dW_qtPQ);
      c->mark("d2h_W");
    }
    c->end_timing();
  });
}

int coqui_b200_set_w(coqui_b200_ctx* c, const double* dW_qtPQ) {
  return guarded(c, [&] {
    require_ready(c, true, true, true);
    CQ_REQUIRE(dW_qtPQ, COQUI_B200_EINVAL, "null W");
    if (c->sym) {
      sym_set_w(c, dW_qtPQ);
      return;
    }
    const int64_t ncol = c->Np * c->Np, n = c->nq * c->nth * ncol;
    c->PW.ensure((size_t)c->nmax * c->nq * ncol * c->elem());
    c->stage.ensure(n);
    upload(c, c->stage.p, dW_qtPQ, n * sizeof(double2));
    if (c->mode == COQUI_B200_FP64)
      cq::launch_qt_to_tq<double>(c->stage.p, (double2*)c->PW.p, c->nth, c->nq, ncol, c->st);
    else
      cq::launch_qt_to_tq<float>(c->stage.p, (float2*)c->PW.p, c->nth, c->nq, ncol, c->st);
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->stage.release();
    c->w_valid = true;
    c->w_in_R = false;
    c->eps_raw_valid = false;
  });
}

int coqui_b200_eval_sigma(coqui_b200_ctx* c, const double* G_tskij, double* Sigma_tskij) {
  return guarded(c, [&] {
    require_ready(c, true, true, true);
    if (c->sym) {
      CQ_REQUIRE(c->sym->w_valid, COQUI_B200_EINVAL,
                 "no screened interaction: call update_w or set_w");
      c->begin_timing();
      sym_upload_g(c, G_tskij);
      c->mark("h2d_G");
      sym_sigma(c, Sigma_tskij);
      c->end_timing();
      return;
    }
    CQ_REQUIRE(c->w_valid, COQUI_B200_EINVAL, "no screened interaction: call update_w or set_w");
    c->begin_timing();
    upload_G(c, G_tskij);
    c->mark("h2d_G");
    sigma_device(c, Sigma_tskij);
    c->end_timing();
  });
}

int coqui_b200_gw_iteration(coqui_b200_ctx* c, const double* G_tskij, double* Sigma_tskij,
                            double* eps_inv_head) {
  return guarded(c, [&] {
    require_ready(c, true, true, true);
    if (c->sym) {
      c->begin_timing();
      sym_upload_g(c, G_tskij);
      c->mark("h2d_G");
      sym_update_w(c);
      if (eps_inv_head) {
        sym_eps_head(c, eps_inv_head);
        c->mark("EPS_INV_HEAD");
      }
      sym_sigma(c, Sigma_tskij);
      c->end_timing();
      return;
    }
    // resident G or page-locked host buffers, no eps head: the iteration (the copies included)
    // runs as one CUDA graph, captured on the first of a run of such calls with the same
    // buffers and replayed by the following ones
    // page-locked host buffers: the copies join the graph
    if (!eps_inv_head && c->mode == COQUI_B200_MIXED && !c->prof.on && !div_active(c) &&
        (G_tskij ? is_pinned(G_tskij) : c->g_resident) && (!Sigma_tskij || is_pinned(Sigma_tskij))) {
      gw_iteration_graph(c, G_tskij, Sigma_tskij);
      return;
    }
    c->begin_timing();
    upload_G(c, G_tskij);
    c->mark("h2d_G");
    // mixed form: no host round trip between the Dyson step and the self-energy; the
    // factorisation status is checked once the iteration has run
    const bool defer = (c->mode == COQUI_B200_MIXED);
    c->defer_dyson_check = defer;
    try {
      update_w_device(c);
      if (eps_inv_head) {
        eps_head(c, eps_inv_head);
        c->mark("EPS_INV_HEAD");
      }
      sigma_device(c, Sigma_tskij);
    } catch (...) {
      c->defer_dyson_check = false;
      throw;
    }
    c->defer_dyson_check = false;
    if (defer) check_dyson_status(c);
    c->end_timing();
  });
}

int coqui_b200_set_profiling(coqui_b200_ctx* c, int on) {
  return guarded(c, [&] {
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->prof.resolve();
    c->prof.acc.clear();
    c->prof.on = (on != 0);
  });
}

int coqui_b200_kernel_stats(const coqui_b200_ctx* c, char* names, int name_len, double* ms,
                            int64_t* launches, int n) {
  if (!c) return COQUI_B200_EINVAL;
  int k = 0;
  for (const auto& p : c->prof.acc) {
    if (k >= n) break;
    if (names && name_len > 0) {
      std::strncpy(names + (size_t)k * name_len, p.first.c_str(), name_len - 1);
      names[(size_t)k * name_len + name_len - 1] = 0;
    }
    if (ms) ms[k] = std::get<0>(p.second);
    if (launches) launches[k] = std::get<1>(p.second);
    ++k;
  }
  return k;
}

int coqui_b200_set_gcache_limit(coqui_b200_ctx* c, int64_t bytes) {
  return guarded(c, [&] {
    CQ_REQUIRE(bytes >= -1, COQUI_B200_EINVAL, "cache limit must be -1, 0 or a byte count");
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    // captured iteration graphs hold the cache's address
    if (c->gexec) {
      cudaGraphExecDestroy(c->gexec);
      c->gexec = nullptr;
    }
    if (c->rexec) {
      cudaGraphExecDestroy(c->rexec);
      c->rexec = nullptr;
    }
    c->gcache_limit = bytes;
    c->Gcache.release();
    c->gcache_valid = false;
    c->gcache_pairs = 0;
  });
}

int coqui_b200_kernel_units(const coqui_b200_ctx* c, char* names, int name_len, int64_t* units,
                            int n) {
  if (!c) return COQUI_B200_EINVAL;
  int k = 0;
  for (const auto& p : c->prof.acc) {
    if (k >= n) break;
    if (names && name_len > 0) {
      std::strncpy(names + (size_t)k * name_len, p.first.c_str(), name_len - 1);
      names[(size_t)k * name_len + name_len - 1] = 0;
    }
    if (units) units[k] = std::get<2>(p.second);
    ++k;
  }
  return k;
}

int coqui_b200_rpa_energy(coqui_b200_ctx* c, const double* G_tskij, double* e_rpa) {
  return guarded(c, [&] {
    require_ready(c, true, true, true);
    CQ_REQUIRE(e_rpa, COQUI_B200_EINVAL, "null e_rpa");
    CQ_REQUIRE(c->Ttw_bb.size() == (size_t)(c->nt * c->nwb), COQUI_B200_EINVAL, "IR tables");
    if (c->sym) {
      *e_rpa = sym_rpa_energy(c, G_tskij);
      return;
    }
    // resident G or a page-locked host G: one CUDA graph, captured on the first of a run of
    // such calls and replayed by the following ones
    if (c->mode == COQUI_B200_MIXED && !c->prof.on &&
        (G_tskij ? is_pinned(G_tskij) : c->g_resident)) {
      rpa_energy_graph(c, G_tskij, e_rpa);
      return;
    }
    c->begin_timing();
    upload_G(c, G_tskij);
    c->mark("h2d_G");
    eval_pi_device(c);
    c->mark("EVALUATE_PI_R");
    ir_inplace(c, (int)c->nth, (int)c->nwh, c->dTwt.p);
    c->mark("IMAG_FT_TtoW");
    std::vector<double> ld;
    std::vector<double2> tr;
    dyson_all(c, false, true, &ld, &tr);
    c->mark("EVALUATE_RPA");
    for (double v : ld)
      CQ_REQUIRE(std::isfinite(v), COQUI_B200_ENOTHPD, "I - Pi V is not positive definite");
    *e_rpa = rpa_energy_from(c, ld, tr);
    c->end_timing();
  });
}

int coqui_b200_tau_to_w(coqui_b200_ctx* c, const double* X_tqPQ, double* X_wqPQ) {
  return guarded(c, [&] {
    require_ready(c, false, true, false);
    CQ_REQUIRE(X_tqPQ && X_wqPQ, COQUI_B200_EINVAL, "null arguments");
    const int64_t ncol = c->nq * c->Np * c->Np;
    c->PW.ensure((size_t)c->nmax * ncol * c->elem());
    c->stage.ensure((size_t)c->nmax * ncol);
    upload(c, c->stage.p, X_tqPQ, (size_t)c->nth * ncol * sizeof(double2));
    if (c->mode == COQUI_B200_FP64)
      CQ_CHECK_CUDA(cudaMemcpyAsync(c->PW.p, c->stage.p, (size_t)c->nth * ncol * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, c->st));
    else
      cq::launch_from_c128<float>(c->stage.p, (float2*)c->PW.p, c->nth * ncol, c->st);
    ir_inplace(c, (int)c->nth, (int)c->nwh, c->dTwt.p);
    if (c->mode == COQUI_B200_FP64)
      download(c, X_wqPQ, c->PW.p, (size_t)c->nwh * ncol * sizeof(double2));
    else {
      cq::launch_to_c128<float>((float2*)c->PW.p, c->stage.p, c->nwh * ncol, c->st);
      download(c, X_wqPQ, c->stage.p, (size_t)c->nwh * ncol * sizeof(double2));
    }
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->w_valid = false;
  });
}

int coqui_b200_w_to_tau(coqui_b200_ctx* c, const double* X_wqPQ, double* X_tqPQ) {
  return guarded(c, [&] {
    require_ready(c, false, true, false);
    CQ_REQUIRE(X_tqPQ && X_wqPQ, COQUI_B200_EINVAL, "null arguments");
    const int64_t ncol = c->nq * c->Np * c->Np;
    c->PW.ensure((size_t)c->nmax * ncol * c->elem());
    c->stage.ensure((size_t)c->nmax * ncol);
    upload(c, c->stage.p, X_wqPQ, (size_t)c->nwh * ncol * sizeof(double2));
    if (c->mode == COQUI_B200_FP64)
      CQ_CHECK_CUDA(cudaMemcpyAsync(c->PW.p, c->stage.p, (size_t)c->nwh * ncol * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, c->st));
    else
      cq::launch_from_c128<float>(c->stage.p, (float2*)c->PW.p, c->nwh * ncol, c->st);
    ir_inplace(c, (int)c->nwh, (int)c->nth, c->dTtw.p);
    if (c->mode == COQUI_B200_FP64)
      download(c, X_tqPQ, c->PW.p, (size_t)c->nth * ncol * sizeof(double2));
    else {
      cq::launch_to_c128<float>((float2*)c->PW.p, c->stage.p, c->nth * ncol, c->st);
      download(c, X_tqPQ, c->stage.p, (size_t)c->nth * ncol * sizeof(double2));
    }
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->w_valid = false;
  });
}

int coqui_b200_dyson_w(coqui_b200_ctx* c, const double* Pi_wqPQ, double* W_wqPQ) {
  return guarded(c, [&] {
    require_ready(c, true, false, false);
    CQ_REQUIRE(Pi_wqPQ && W_wqPQ, COQUI_B200_EINVAL, "null arguments");
    // one frequency at a time: reuse the PW buffer with nw = 1 slabs
    const int64_t ncol = c->nq * c->Np * c->Np;
    const int64_t nw = c->nwh;
    c->PW.ensure((size_t)c->nmax * ncol * c->elem());
    c->stage.ensure((size_t)nw * ncol);
    upload(c, c->stage.p, Pi_wqPQ, (size_t)nw * ncol * sizeof(double2));
    if (c->mode == COQUI_B200_FP64)
      CQ_CHECK_CUDA(cudaMemcpyAsync(c->PW.p, c->stage.p, (size_t)nw * ncol * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, c->st));
    else
      cq::launch_from_c128<float>(c->stage.p, (float2*)c->PW.p, nw * ncol, c->st);
    dyson_all(c, true, false, nullptr, nullptr);
    if (c->mode == COQUI_B200_FP64)
      download(c, W_wqPQ, c->PW.p, (size_t)nw * ncol * sizeof(double2));
    else {
      cq::launch_to_c128<float>((float2*)c->PW.p, c->stage.p, nw * ncol, c->st);
      download(c, W_wqPQ, c->stage.p, (size_t)nw * ncol * sizeof(double2));
    }
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->w_valid = false;
  });
}


int coqui_b200_set_ir_fermi(coqui_b200_ctx* c, const double* Twt_ff, const double* Ttw_ff,
                            const int64_t* wn_mesh_f, int64_t nw_f, double beta) {
  return guarded(c, [&] {
    CQ_REQUIRE(Twt_ff && Ttw_ff && wn_mesh_f && nw_f >= 1 && beta > 0, COQUI_B200_EINVAL,
               "bad fermionic IR tables");
    const int64_t nt = c->nt;
    c->nwf = nw_f;
    c->beta = beta;
    c->wnf.assign(wn_mesh_f, wn_mesh_f + nw_f);
    c->Ttw_ff_h.resize(nt * nw_f);
    for (int64_t i = 0; i < nt * nw_f; ++i) c->Ttw_ff_h[i] = make_double2(Ttw_ff[2 * i], Ttw_ff[2 * i + 1]);
    c->dTwt_ff.ensure(nw_f * nt);
    c->dTtw_ff.ensure(nt * nw_f);
    c->dwnf.ensure(nw_f);
    upload(c, c->dTwt_ff.p, Twt_ff, nw_f * nt * sizeof(double2));
    upload(c, c->dTtw_ff.p, Ttw_ff, nt * nw_f * sizeof(double2));
    upload(c, c->dwnf.p, wn_mesh_f, nw_f * sizeof(int64_t));
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->have_irf = true;
  });
}

int coqui_b200_set_mean_field(coqui_b200_ctx* c, const double* H0_skij, const double* S_skij,
                              const double* F_skij, double mu) {
  return guarded(c, [&] {
    CQ_REQUIRE(H0_skij && S_skij && F_skij, COQUI_B200_EINVAL, "null mean-field arrays");
    const int64_t n = c->nk * c->nb * c->nb;
    for (auto* b : {&c->H0, &c->Sov, &c->F, &c->F_mf}) b->ensure(n);
    upload(c, c->H0.p, H0_skij, n * sizeof(double2));
    upload(c, c->Sov.p, S_skij, n * sizeof(double2));
    upload(c, c->F.p, F_skij, n * sizeof(double2));
    upload(c, c->F_mf.p, F_skij, n * sizeof(double2));
    CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
    c->mu = mu;
    c->have_mf = true;
    c->dx.clear();
    c->dr.clear();
    c->dB.clear();
  });
}

int coqui_b200_set_iter_alg(coqui_b200_ctx* c, int alg, double mixing, int64_t max_subsp,
                            int64_t diis_start) {
  return guarded(c, [&] {
    CQ_REQUIRE((alg == 0 || alg == 1) && mixing > 0 && mixing <= 1 && max_subsp >= 2,
               COQUI_B200_EINVAL, "bad iteration parameters");
    c->iter_alg = alg;
    c->mixing = mixing;
    c->max_subsp = max_subsp;
    c->diis_start = diis_start;
  });
}

int coqui_b200_set_div_treatment(coqui_b200_ctx* c, int div_treatment, double madelung,
                                 const double* chi_head_P) {
  return guarded(c, [&] {
    CQ_REQUIRE(div_treatment >= 0 && div_treatment <= 3, COQUI_B200_EINVAL,
               "div_treatment must be 0 (ignore_g0), 1 (gygi), 2 (gygi_extrplt) or "
               "3 (gygi_extrplt_2d)");
    c->div = div_treatment;
    c->madelung = madelung;
    if (chi_head_P) {
      std::vector<double2> h(c->Np);
      std::memcpy(h.data(), chi_head_P, c->Np * sizeof(double2));
      for (auto& v : h) v.y = -v.y;  // conj(chi_head), thc_gw.icc:485
      c->chi0c.ensure(c->Np);
      upload(c, c->chi0c.p, h.data(), c->Np * sizeof(double2));
      CQ_CHECK_CUDA(cudaStreamSynchronize(c->st));
      c->tdiv_valid = false;
    }
  });
}

int coqui_b200_hf_evaluate(coqui_b200_ctx* c, const double* Dm_skij, const double* S_skij,
                           int hartree, int exchange, int div_treatment, double madelung,
                           double* F_skij) {
  return guarded(c, [&] {
    require_ready(c, true, false, true);
    CQ_REQUIRE(Dm_skij && F_skij, COQUI_B200_EINVAL, "null density or Fock matrix");
    CQ_REQUIRE(div_treatment == 0 || div_treatment == 1, COQUI_B200_EINVAL,
               "div_treatment must be 0 (ignore_g0) or 1 (gygi)");
    const bool gygi = exchange && div_treatment == 1;
    CQ_REQUIRE(!gygi || S_skij, COQUI_B200_EINVAL, "gygi needs the overlap matrix");
    const int64_t n = c->nk * c->nb * c->nb;
    c->begin_timing();
    c->hfd.ensure(n);
    c->hff.ensure(n);
    upload(c, c->hfd.p, Dm_skij, n * sizeof(double2));
    if (gygi) {
      c->hfs.ensure(n);
      upload(c, c->hfs.p, S_skij, n * sizeof(double2));
    }
    c->mark("h2d_Dm");
    hf_device(c, c->hfd.p, gygi ? c->hfs.p : nullptr, hartree != 0, exchange != 0,
              div_treatment, madelung, c->hff.p);
    c->mark("HF");
    download(c, F_skij, c->hff.p, n * sizeof(double2));
    c->mark("d2h_F");
    c->end_timing();
  });
}

int coqui_b200_scgw_set_hf(coqui_b200_ctx* c, int enable, int div_treatment, double madelung) {
  return guarded(c, [&] {
    CQ_REQUIRE(div_treatment == 0 || div_treatment == 1, COQUI_B200_EINVAL,
               "div_treatment must be 0 (ignore_g0) or 1 (gygi)");
    c->hf_on = enable != 0;
    c->hf_div = div_treatment;
    c->hf_madelung = madelung;
  });
}

int coqui_b200_scgw_iteration(coqui_b200_ctx* c, const double* G_tskij, int64_t it, double* stats) {
  return guarded(c, [&] {
    require_scgw(c);
    CQ_REQUIRE(it >= 1 && stats, COQUI_B200_EINVAL, "bad iteration arguments");
    const int64_t nF = c->nk * c->nb * c->nb, nS = c->nt * nF;
    CQ_REQUIRE(it == 1 || c->prevFS.n >= (size_t)(nF + nS), COQUI_B200_EINVAL,
               "iteration > 1 without a previous iteration");
    c->begin_timing();
    upload_G(c, G_tskij);
    // the DIIS copy and the density matrix below read all of G: a page-locked G that is
    // still arriving in chunks on the copy stream must have landed first
    for (int64_t i = 0; i < n_tau_chunks(c); ++i) wait_G_chunk(c, i);
    c->mark("h2d_G");
    if (c->iter_alg == 1) {  // the residual of this step is taken with the incoming G
      c->Gin.ensure(nS);
      CQ_CHECK_CUDA(cudaMemcpyAsync(c->Gin.p, c->G.p, nS * sizeof(double2),
                                    cudaMemcpyDeviceToDevice, c->st));
    }
    if (c->hf_on) {  // scf_driver.cpp:94-114: F = J + K of the current density matrix
      if (it == 1) dm_from_g(c);
      hf_device(c, c->Dm.p, c->Sov.p, true, true, c->hf_div, c->hf_madelung, c->F.p);
      c->mark("HF");
    }
    update_w_device(c);
    sigma_device(c, nullptr);
    // scf_driver.cpp:126-129
    cq::hermitize_c128(c->F.p, c->nb, c->nk, c->st);
    cq::hermitize_c128(c->Sig.p, c->nb, c->nt * c->nk, c->st);
    c->FS.ensure(nF + nS);
    CQ_CHECK_CUDA(cudaMemcpyAsync(c->FS.p, c->F.p, nF * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(c->FS.p + nF, c->Sig.p, nS * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, c->st));
    double cF = 0, cS = 0, resid = 0;
    int flag = 0, evals = 1;
    {
      cq::Prof::Scope sc(&c->prof, "scgw_iterate");
      if (it == 1) {  // solve_iterative, it == 1 (scf_common.cpp:320-347)
        cF = cq::maxabs_diff(c->F_mf.p, c->FS.p, nF, c->red, c->st);
        cS = cq::maxabs_diff(c->FS.p + nF, nullptr, nS, c->red, c->st);
        c->dx.clear();
        c->dr.clear();
        c->dB.clear();
        if (c->iter_alg == 1) {
          auto x = std::make_unique<DevBuf<double2>>();
          x->ensure(nF + nS);
          CQ_CHECK_CUDA(cudaMemcpyAsync(x->p, c->FS.p, (nF + nS) * sizeof(double2),
                                        cudaMemcpyDeviceToDevice, c->st));
          c->dx.push_back(std::move(x));
        }
        resid = cS;
        c->r_prev = cS;
        c->nhist = 0;
        c->last_mlp = false;
        c->cooldown = 0;
        if (c->mlp_on) push_history(c, c->FS.p + nF);
      } else if (c->iter_alg == 0) {  // damp_t (damp_t.hpp:34-57)
        resid = cq::maxabs_diff(c->prevFS.p + nF, c->FS.p + nF, nS, c->red, c->st);
        if (c->mlp_on && c->last_mlp && resid > c->r_prev) {
          // the learned proposal raised the residual: evaluate the plain damped Sigma instead
          CQ_CHECK_CUDA(cudaMemcpyAsync(c->prevFS.p + nF, c->plain_saved.p, nS * sizeof(double2),
                                        cudaMemcpyDeviceToDevice, c->st));
          dyson_g_device(c, c->prevFS.p + nF);
          update_w_device(c);
          sigma_device(c, nullptr);
          cq::hermitize_c128(c->Sig.p, c->nb, c->nt * c->nk, c->st);
          CQ_CHECK_CUDA(cudaMemcpyAsync(c->FS.p + nF, c->Sig.p, nS * sizeof(double2),
                                        cudaMemcpyDeviceToDevice, c->st));
          resid = cq::maxabs_diff(c->prevFS.p + nF, c->FS.p + nF, nS, c->red, c->st);
          c->cooldown = 3;
          c->nhist = 0;
          flag = -1;
          ++evals;
        }
        const double m = c->mixing;
        cq::axpby_c128(c->prevFS.p, c->FS.p, 1.0 - m, m, nF + nS, c->st);
        cF = cq::maxabs_diff(c->prevFS.p, c->FS.p, nF, c->red, c->st);
        cS = cq::maxabs_diff(c->prevFS.p + nF, c->FS.p + nF, nS, c->red, c->st);
        if (c->mlp_on) {
          push_history(c, c->FS.p + nF);
          c->last_mlp = false;
          if (c->cooldown > 0) {
            --c->cooldown;
          } else if (c->nhist == 4) {
            const int64_t nel = c->nwf * c->nk * c->nb;
            c->plain_saved.ensure(nS);
            CQ_CHECK_CUDA(cudaMemcpyAsync(c->plain_saved.p, c->FS.p + nF, nS * sizeof(double2),
                                          cudaMemcpyDeviceToDevice, c->st));
            double2* delta = c->dhist.p + 4 * nel;  // fifth slot of the history buffer
            cq::mlp_extrapolate(mlp_net(c->mlp), c->dhist.p, nel, c->mlp_max_jump, delta, c->st);
            add_diag_w(c, delta, c->FS.p + nF);
            c->last_mlp = true;
            c->nhist = 0;
            if (flag == 0) flag = 1;
          }
          c->r_prev = resid;
        }
      } else {
        resid = cq::maxabs_diff(c->prevFS.p + nF, c->FS.p + nF, nS, c->red, c->st);
        std::tie(cF, cS) = diis_device(c, c->FS.p, it);
      }
    }
    CQ_CHECK_CUDA(cudaMemcpyAsync(c->F.p, c->FS.p, nF * sizeof(double2), cudaMemcpyDeviceToDevice, c->st));
    CQ_CHECK_CUDA(cudaMemcpyAsync(c->Sig.p, c->FS.p + nF, nS * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, c->st));
    c->prevFS.ensure(nF + nS);
    CQ_CHECK_CUDA(cudaMemcpyAsync(c->prevFS.p, c->FS.p, (nF + nS) * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, c->st));
    c->mark("ITERATIVE");
    dyson_g_device(c, c->Sig.p);
    c->mark("DYSON");
    double e1 = 0, ehf = 0;
    hf_energy_device(c, &e1, &ehf);
    const double ec = gm_energy_device(c, c->G.p, c->Sig.p);
    c->mark("ENERGIES");
    stats[0] = cF;
    stats[1] = cS;
    stats[2] = e1;
    stats[3] = ehf;
    stats[4] = ec;
    stats[5] = resid;
    stats[6] = flag;
    stats[7] = evals;
    c->end_timing();
  });
}

int coqui_b200_scgw_set_mlp(coqui_b200_ctx* c, coqui_b200_mlp* mlp, int enable, double max_jump) {
  return guarded(c, [&] {
    CQ_REQUIRE(!enable || (mlp && max_jump > 0), COQUI_B200_EINVAL, "enable needs an mlp");
    if (enable) CQ_REQUIRE(mlp_net(mlp).din == 4 && mlp_net(mlp).dout == 2, COQUI_B200_EINVAL,
                           "the learned update takes a network with 4 inputs and 2 outputs");
    c->mlp = enable ? mlp : nullptr;
    c->mlp_on = enable != 0;
    c->mlp_max_jump = max_jump;
    c->nhist = 0;
    c->last_mlp = false;
    c->cooldown = 0;
  });
}

int coqui_b200_scgw_sigma_diag_w(coqui_b200_ctx* c, double* out) {
  return guarded(c, [&] {
    CQ_REQUIRE(c->have_irf && out, COQUI_B200_EINVAL, "bad arguments (set_ir_fermi first)");
    const int64_t nS = c->nt * c->nk * c->nb * c->nb, nel = c->nwf * c->nk * c->nb;
    CQ_REQUIRE(c->Sig.n >= (size_t)nS, COQUI_B200_EINVAL, "no self-energy yet");
    c->trc.ensure(nel);
    sigma_diag_w(c, c->Sig.p, c->trc.p);
    download(c, out, c->trc.p, nel * sizeof(double2));
  });
}

int coqui_b200_get_scgw_state(coqui_b200_ctx* c, double* G_tskij, double* Sigma_tskij,
                              double* Dm_skij) {
  return guarded(c, [&] {
    const int64_t nF = c->nk * c->nb * c->nb, nS = c->nt * nF;
    if (G_tskij) {
      CQ_REQUIRE(c->g_resident && c->G.n >= (size_t)nS, COQUI_B200_EINVAL, "no resident G");
      download(c, G_tskij, c->G.p, nS * sizeof(double2));
    }
    if (Sigma_tskij) {
      CQ_REQUIRE(c->Sig.n >= (size_t)nS, COQUI_B200_EINVAL, "no self-energy yet");
      download(c, Sigma_tskij, c->Sig.p, nS * sizeof(double2));
    }
    if (Dm_skij) {
      CQ_REQUIRE(c->Dm.n >= (size_t)nF, COQUI_B200_EINVAL, "no density matrix yet");
      download(c, Dm_skij, c->Dm.p, nF * sizeof(double2));
    }
  });
}

int coqui_b200_dyson_g(coqui_b200_ctx* c, const double* Sigma_tskij, double* G_tskij,
                       double* Dm_skij) {
  return guarded(c, [&] {
    require_scgw(c);
    CQ_REQUIRE(Sigma_tskij, COQUI_B200_EINVAL, "null Sigma");
    const int64_t nF = c->nk * c->nb * c->nb, nS = c->nt * nF;
    c->Sig.ensure(nS);
    upload(c, c->Sig.p, Sigma_tskij, nS * sizeof(double2));
    dyson_g_device(c, c->Sig.p);
    if (G_tskij) download(c, G_tskij, c->G.p, nS * sizeof(double2));
    if (Dm_skij) download(c, Dm_skij, c->Dm.p, nF * sizeof(double2));
  });
}

int coqui_b200_gm_energy(coqui_b200_ctx* c, const double* G_tskij, const double* Sigma_tskij,
                         double* e_corr) {
  return guarded(c, [&] {
    CQ_REQUIRE(c->have_irf && G_tskij && Sigma_tskij && e_corr, COQUI_B200_EINVAL,
               "bad arguments (set_ir_fermi first)");
    const int64_t nS = c->nt * c->nk * c->nb * c->nb;
    c->stage.ensure(2 * nS);
    upload(c, c->stage.p, G_tskij, nS * sizeof(double2));
    upload(c, c->stage.p + nS, Sigma_tskij, nS * sizeof(double2));
    *e_corr = gm_energy_device(c, c->stage.p, c->stage.p + nS);
  });
}

void coqui_b200_set_autotune(int on) { cq::tc_set_autotune(on); }

int64_t coqui_b200_tuned_shapes(void) { return cq::tc_tuned_shapes(); }

int coqui_b200_set_tile_config(int cfg) {
  return cq::tc_set_forced_cfg(cfg) ? COQUI_B200_OK : COQUI_B200_EINVAL;
}

int coqui_b200_num_tile_configs(void) { return cq::tc_num_cfgs(); }

int coqui_b200_factor_dielectric(const float* M_dev, double* A_dev, double* logdet_dev,
                                 double* trace_dev, int* info_dev, int64_t Np, int64_t nprob,
                                 void* stream) {
  try {
    CQ_REQUIRE(M_dev && A_dev && logdet_dev && trace_dev && info_dev, COQUI_B200_EINVAL,
               "factor_dielectric: null argument");
    CQ_REQUIRE(Np > 0 && nprob > 0 && nprob <= 2147483647, COQUI_B200_EINVAL,
               "factor_dielectric: bad sizes");
    const void* ptrs[] = {M_dev, A_dev, logdet_dev, trace_dev, info_dev};
    int dev = -1;
    for (const void* q : ptrs) {
      cudaPointerAttributes at{};
      CQ_CHECK_CUDA(cudaPointerGetAttributes(&at, q));
      CQ_REQUIRE(at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged,
                 COQUI_B200_EINVAL, "factor_dielectric: arguments must be device memory");
      CQ_REQUIRE(dev < 0 || at.device == dev, COQUI_B200_EINVAL,
                 "factor_dielectric: arguments on different devices");
      dev = at.device;
    }
    CQ_CHECK_CUDA(cudaSetDevice(dev));
    cudaStream_t st = (cudaStream_t)stream;
    cq::launch_chol_group_inv(reinterpret_cast<const float2*>(M_dev),
                              reinterpret_cast<double2*>(A_dev), logdet_dev,
                              reinterpret_cast<double2*>(trace_dev), info_dev, Np, nprob, st);
    CQ_CHECK_CUDA(cudaStreamSynchronize(st));
    return COQUI_B200_OK;
  } catch (const cq::Error& e) {
    return e.code;
  }
}

int coqui_b200_set_wait_limit_ns(int device, int64_t ns) {
  try {
    CQ_CHECK_CUDA(cudaSetDevice(device));
    cq::tc_set_wait_ns(ns);
    return COQUI_B200_OK;
  } catch (const cq::Error& e) {
    return e.code;
  }
}

}  // extern "C"
