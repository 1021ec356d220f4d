/*
 * coqui_b200.h -- C ABI of the B200 THC-RPA/GW imaginary-time hot path.
 *
 * One context (coqui_b200_ctx) holds the THC data, the IR grids, the k-mesh and every
 * device buffer of one system.  The entry points mirror CoQui's solver entry points
 * on this path (paths relative to the CoQui tree):
 *
 *   coqui_b200_update_w     <- methods::solvers::scr_coulomb_t::update_w
 *                              (src/methods/scr_coulomb/scr_coulomb_t.cpp:37-95)
 *   coqui_b200_eval_sigma   <- methods::solvers::gw_t::evaluate(MBState&, THC_ERI const&)
 *                              (src/methods/GW/thc_gw.cpp:26-89, thc_gw.icc:70-213)
 *   coqui_b200_rpa_energy   <- methods::solvers::gw_t::rpa_energy / thc_rpa_Xqindep
 *                              (src/methods/GW/thc_rpa.cpp:22, thc_rpa.icc:21-181)
 *   coqui_b200_eval_pi      <- scr_coulomb_t::eval_Pi_qdep -> eval_Pi_rpa_Rspace
 *                              (scr_coulomb_t.cpp:262-280, rpa_pi.icc:22-180)
 *   coqui_b200_primary_to_aux / coqui_b200_aux_to_primary
 *                           <- thc_solver_comm::primary_to_aux / aux_to_primary
 *                              (src/methods/HF/thc_solver_comm.hpp:363-429, 516-569)
 *   coqui_b200_tau_to_w / coqui_b200_w_to_tau
 *                           <- scr_coulomb_t::tau_to_w / w_to_tau (PH-symmetric IR)
 *                              (scr_coulomb_t.cpp:349-488, IAFT.icc:49-128)
 *   coqui_b200_dyson_w      <- scr_coulomb_t::dyson_W_in_place (scr_coulomb_t.cpp:121-206)
 *   coqui_b200_set_thc      <- thc_reader_t::X(is,ip,ik) / Z(iq,...) data
 *                              (src/methods/ERI/thc_reader_t.hpp:590-604, 714-751)
 *   coqui_b200_set_ir       <- imag_axes_ft::ir::IR tables (ir/ir_driver.hpp:23-76)
 *   coqui_b200_set_kmesh    <- mf::MF kpts/lattv/kp_grid (src/mean_field/MF.hpp:152-247)
 *
 * Conventions (kept from the reference):
 *   - host arrays are C-ordered and caller-owned; complex values are complex128 stored
 *     as (re, im) double pairs;
 *   - G_tskij and Sigma_tskij are (nt_f, ns, nk, nb, nb); X is (ns, nk, Np, nb);
 *     V is (nq, Np, Np); W is returned as dW_qtPQ (nq, nt_half, Np, Np);
 *   - Sigma is overwritten (thc_gw.cpp:136);
 *   - X and V cover the whole k-mesh, nq == nk, k-points form a Gamma-centred kp_grid in
 *     lexicographic order (kpts = 2 pi (i,j,l)/n in units where lattv rows are the lattice
 *     vectors); after coqui_b200_set_symmetry, G, Sigma, Pi and W cover the IBZ points.
 * Errors: every entry point returns 0 or a negative COQUI_B200_E* code and never aborts;
 * coqui_b200_last_error() gives the message.  One host thread per context; calls are
 * synchronous (they return after the device work finished).
 */
#ifndef COQUI_B200_H
#define COQUI_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define COQUI_B200_API __attribute__((visibility("default")))
#else
#define COQUI_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define COQUI_B200_OK 0
#define COQUI_B200_EINVAL -1       /* bad argument, shape or order of calls */
#define COQUI_B200_EUNSUPPORTED -2 /* input outside the supported domain (e.g. k-mesh order) */
#define COQUI_B200_ECUDA -3        /* CUDA runtime / library error */
#define COQUI_B200_ENOMEM -4       /* device allocation failed */
#define COQUI_B200_ENOTHPD -5      /* a matrix that must be Hermitian positive definite is not */
#define COQUI_B200_EPHSYM -6       /* tau mesh not particle-hole symmetric (thc_gw.cpp:56-66) */
#define COQUI_B200_ETIMEDOUT -7    /* a bounded device-side wait gave up */

/* precision_mode */
#define COQUI_B200_FP64 0  /* complex128 everywhere: FP64 tensor-core GEMMs + factorizations */
#define COQUI_B200_MIXED 1 /* split-TF32 tensor-core products, complex64 intermediates,
                              FP64 Cholesky / log-det */

typedef struct coqui_b200_ctx coqui_b200_ctx;
typedef struct coqui_b200_mlp coqui_b200_mlp; /* network of the learned self-energy update */

typedef struct {
  int64_t ns;          /* spin components (1 supported) */
  int64_t nk;          /* k-points (= nq, no symmetry) */
  int64_t nb;          /* orbitals */
  int64_t Np;          /* THC interpolating points N_mu */
  int64_t nt_f;        /* fermionic tau points */
  int64_t nw_b;        /* bosonic Matsubara points */
  int64_t kp_grid[3];  /* Monkhorst-Pack grid */
  int32_t precision_mode;
  int32_t device;      /* CUDA device ordinal */
} coqui_b200_dims;

COQUI_B200_API int coqui_b200_create(coqui_b200_ctx** ctx, const coqui_b200_dims* dims);
COQUI_B200_API void coqui_b200_destroy(coqui_b200_ctx* ctx);
COQUI_B200_API const char* coqui_b200_last_error(const coqui_b200_ctx* ctx);
COQUI_B200_API const char* coqui_b200_version(void);

/* IR tables, already rescaled by beta as in ir_driver.hpp:68-73; complex128 (re,im).
   Twt_bb: (nw_b, nt_b), Ttw_bb: (nt_b, nw_b), T_beta_t_ff: (nt_f),
   tau_mesh_x: (nt_f) in [-1, 1] (checked for particle-hole symmetry). */
COQUI_B200_API int coqui_b200_set_ir(coqui_b200_ctx* ctx, const double* Twt_bb, const double* Ttw_bb,
                      const double* T_beta_t_ff, const double* tau_mesh_x);

/* kpts (nk,3) cartesian, lattv (3,3) rows = lattice vectors; chi_bar_qP (nq, Np) complex
   (may be NULL: dielectric head is then zero). */
COQUI_B200_API int coqui_b200_set_kmesh(coqui_b200_ctx* ctx, const double* kpts, const double* lattv,
                         const double* chi_bar_qP);

/* X_skPa complex128 (ns, nk, Np, nb); V_qPQ complex128 (nq, Np, Np), Hermitian PD. */
COQUI_B200_API int coqui_b200_set_thc(coqui_b200_ctx* ctx, const double* X_skPa, const double* V_qPQ);

/* Pi(tau) in the auxiliary basis: Pi_tqPQ (nt_half, nq, Np, Np) complex128. */
COQUI_B200_API int coqui_b200_eval_pi(coqui_b200_ctx* ctx, const double* G_tskij, double* Pi_tqPQ);

/* Screened interaction.  W kept on the device for coqui_b200_eval_sigma; copied out to
   dW_qtPQ (nq, nt_half, Np, Np) if non-NULL; eps_inv_head (nt_half) complex if non-NULL. */
COQUI_B200_API int coqui_b200_update_w(coqui_b200_ctx* ctx, const double* G_tskij, double* dW_qtPQ,
                        double* eps_inv_head);

/* Self-energy from G and the device-resident W of the last update_w (or set_w).
   G_tskij == NULL (here and in eval_pi, update_w, rpa_energy, gw_iteration) reuses the G that
   the previous call of this context left on the device; after update_w of that G the
   self-energy then also reuses the auxiliary-basis G(tau) that the polarizability formed,
   instead of copying G in and projecting it again. */
COQUI_B200_API int coqui_b200_eval_sigma(coqui_b200_ctx* ctx, const double* G_tskij, double* Sigma_tskij);

/* Upload a screened interaction dW_qtPQ (nq, nt_half, Np, Np) for eval_sigma. */
COQUI_B200_API int coqui_b200_set_w(coqui_b200_ctx* ctx, const double* dW_qtPQ);

/* RPA correlation energy (Ha).  G_tskij == NULL reuses the device-resident G. */
COQUI_B200_API int coqui_b200_rpa_energy(coqui_b200_ctx* ctx, const double* G_tskij, double* e_rpa);

/* One GW iteration of scf_loop (src/methods/SCF/scf_driver.cpp:119-122): update_w then
   gw_t::evaluate.  G_tskij == NULL reuses the device-resident G; Sigma_tskij == NULL keeps
   Sigma on the device; eps_inv_head (nt_half complex) may be NULL.  W stays on the device. */
COQUI_B200_API int coqui_b200_gw_iteration(coqui_b200_ctx* ctx, const double* G_tskij,
                                           double* Sigma_tskij, double* eps_inv_head);

/* ---- long-wavelength (q -> 0) treatment of scr_coulomb_t and gw_t (div_treatment_e) ---- */

/* div_treatment 0 = ignore_g0 (default), 1 = gygi, 2 = gygi_extrplt, 3 = gygi_extrplt_2d.
   The eps^-1 head (update_w, gw_iteration) follows eps_inv_head_t
   (src/methods/GW/g0_div_utils.hpp:55-111): the smallest nonzero |q| for 0 and 1; for 2 and 3
   a quadratic in |q| fitted per bosonic frequency through the q with 0 < |q| <= 0.8 (q_z = 0
   for 3) and extrapolated to q = 0.  For 1-3 the self-energy also gets Sigma_div_correction
   (src/methods/GW/thc_gw.icc:446-526): -madelung Re head(tau) T G(tau) T^H with
   T = X^H diag(conj chi_head) X; chi_head_P is basis_head at q = 0 (Np complex128; needed
   before the first such Sigma, NULL keeps the last one).  With one q-point every treatment
   acts as ignore_g0, as in the reference. */
COQUI_B200_API int coqui_b200_set_div_treatment(coqui_b200_ctx* ctx, int div_treatment,
                                                double madelung, const double* chi_head_P);

/* ---- symmetry-reduced (IBZ) k-space path: scr_coulomb_t::eval_Pi_rpa_kspace
   (src/methods/scr_coulomb/rpa_pi.icc:182-336), gw_t::eval_Sigma_all_kspace
   (src/methods/GW/thc_gw.icc:216-443, selected by thc_gw.icc:31-32 when nqpts_ibz < nqpts)
   and the IBZ-weighted RPA energy (src/methods/GW/thc_rpa.icc:130-173) ---- */

/* The mean field's bz_symm maps (src/mean_field/symmetry/bz_symmetry.hpp), indexed as the
   reference indexes them: its k list (IBZ points first, their time-reversal images last) and
   Qpts = kpts (Gamma-centred grid).  k_lex[i] is the position of the reference's k-point i in
   the lexicographic grid that set_kmesh and set_thc use (X and V stay in that order).
   Qs is (nsym, ld_Qs) with row s holding nq_per_s[s] q indices; ks_to_k is (nsym, nk);
   D is symmetry_rotation(isym, k) as dense (nsym, nk_ibz, nb, nb) complex128 (row 0, the
   identity operation, is not read; NULL: every rotation is the identity). */
typedef struct {
  int64_t nk_ibz;               /* IBZ k-points: the reference's k indices [0, nk_ibz) */
  int64_t nq_ibz;               /* IBZ q-points: the reference's q indices [0, nq_ibz) */
  int64_t nsym;                 /* qsymms.size() */
  int64_t ld_Qs;                /* row length of Qs */
  const int64_t* k_lex;         /* (nk) */
  const int64_t* kp_to_ibz;     /* (nk) */
  const int32_t* kp_trev;       /* (nk) 0 / 1 */
  const int64_t* kp_trev_pair;  /* (nk), -1 where there is none */
  const int64_t* qp_to_ibz;     /* (nq) */
  const int32_t* qp_trev;       /* (nq) 0 / 1 */
  const int64_t* qminus;        /* (nq) */
  const int64_t* nq_per_s;      /* (nsym) */
  const int64_t* Qs;            /* (nsym, ld_Qs) */
  const int64_t* ks_to_k;       /* (nsym, nk) */
  const double* D;              /* (nsym, nk_ibz, nb, nb) complex128 or NULL */
} coqui_b200_symmetry;

/* Checks the maps against the grid of set_kmesh (ranges, IBZ first, time-reversal pairs at -k,
   qminus, every q in exactly one Qs row) and switches the context to the k-space path:
   eval_pi, update_w, set_w, eval_sigma, gw_iteration and rpa_energy then take G_tskij and
   return Sigma_tskij on the IBZ k-points (nt_f, ns, nk_ibz, nb, nb) and Pi / W on the IBZ
   q-points (nt_half, nq_ibz, Np, Np) / dW_qtPQ (nq_ibz, nt_half, Np, Np); G must be given
   (no resident G).  The eps^-1 head runs over the IBZ q-points (eps_inv_head_t with
   Qpts_ibz) and Sigma_div_correction over the IBZ k-points, as in the reference.
   sym == NULL returns to the full-BZ path.  Needs set_kmesh. */
COQUI_B200_API int coqui_b200_set_symmetry(coqui_b200_ctx* ctx, const coqui_b200_symmetry* sym);

/* ---- THC Hartree-Fock (hf_t::evaluate, src/methods/HF/thc_hf.cpp:21-60 ->
   thc_hf.icc:17-272 for q-independent THC without symmetry; hf_t.cpp:45-84) ---- */

/* F_skij (ns, nk, nb, nb) complex128, overwritten, = J (hartree != 0) + K (exchange != 0) of the
   density matrix Dm_skij (ns, nk, nb, nb) with the context's X and V.  div_treatment 0 =
   ignore_g0, 1 = gygi: K also gets -madelung S Dm S (S_skij needed then; may be NULL
   otherwise).  Needs set_thc and set_kmesh. */
COQUI_B200_API int coqui_b200_hf_evaluate(coqui_b200_ctx* ctx, const double* Dm_skij,
                                          const double* S_skij, int hartree, int exchange,
                                          int div_treatment, double madelung, double* F_skij);

/* ---- self-consistent GW loop (scf_loop, src/methods/SCF/scf_driver.cpp:90-173, for GW with a
   constant chemical potential; hf = nullptr unless coqui_b200_scgw_set_hf enables it) ---- */

/* Fermionic IR tables, rescaled by beta as in ir_driver.hpp:68-73: Twt_ff (nw_f, nt_f) and
   Ttw_ff (nt_f, nw_f) complex128, wn_mesh_f (nw_f) Matsubara integers (omega_n = pi wn / beta,
   IAFT.hpp:55-57). */
COQUI_B200_API int coqui_b200_set_ir_fermi(coqui_b200_ctx* ctx, const double* Twt_ff,
                                           const double* Ttw_ff, const int64_t* wn_mesh_f,
                                           int64_t nw_f, double beta);

/* Mean field of the loop: H0_skij, S_skij, F_skij (ns, nk, nb, nb) complex128 (F without H0;
   kept fixed as with hf = nullptr unless coqui_b200_scgw_set_hf enables it) and the chemical
   potential mu. */
COQUI_B200_API int coqui_b200_set_mean_field(coqui_b200_ctx* ctx, const double* H0_skij,
                                             const double* S_skij, const double* F_skij, double mu);

/* Iteration algorithm of solve_iterative (scf_common.cpp:229-355): alg 0 = damping
   (damp_t.hpp:34-48, mixing), 1 = commutator DIIS (diis_t.hpp:58-100; mixing of its damping
   steps, max_subsp, diis_start). */
COQUI_B200_API int coqui_b200_set_iter_alg(coqui_b200_ctx* ctx, int alg, double mixing,
                                           int64_t max_subsp, int64_t diis_start);

/* enable != 0: every iteration first re-evaluates F = J + K (+ the gygi term with the
   mean-field overlap) from the density matrix, as scf_loop does with an hf solver
   (scf_driver.cpp:94-114); iteration 1 takes Dm = -G(beta^-) of the starting G. */
COQUI_B200_API int coqui_b200_scgw_set_hf(coqui_b200_ctx* ctx, int enable, int div_treatment,
                                          double madelung);

/* One loop iteration it (>= 1): [HF,] update_w, Sigma, hermitize, damping/DIIS, Dyson for G
   (simple_dyson.cpp:11-123, G stays resident for the next iteration), energies.
   G_tskij != NULL uploads the starting G (iteration 1).  stats[8] = max|dF|, max|dSigma|,
   e_1e, e_hf, e_corr (Galitskii-Migdal, scf_common.cpp:87-136), the residual
   max|Sigma_GW - Sigma_in| of this iteration, learned-update flag (1 applied, -1 withdrawn
   and re-evaluated, 0 none), number of GW evaluations in this call. */
COQUI_B200_API int coqui_b200_scgw_iteration(coqui_b200_ctx* ctx, const double* G_tskij,
                                             int64_t it, double* stats);

/* Learned update of the damped loop (alg 0): after the damping step, the network extrapolates
   every diagonal element Sigma_ii^k(i w_n) from its last four iterates and the loop adds the
   proposal (back on the tau grid, made Hermitian).  The next iteration judges it by the
   residual max|Sigma_GW - Sigma_in|: if that grew, the proposal is withdrawn, the plain damped
   Sigma is evaluated instead and the network pauses for three iterations.  mlp NULL or enable 0
   switches it off.  The mlp must outlive its use by the context. */
COQUI_B200_API int coqui_b200_scgw_set_mlp(coqui_b200_ctx* ctx, coqui_b200_mlp* mlp, int enable,
                                           double max_jump);

/* Diagonal of the current loop self-energy on the fermionic frequency grid:
   out (nw_f, nk, nb) complex128. */
COQUI_B200_API int coqui_b200_scgw_sigma_diag_w(coqui_b200_ctx* ctx, double* out);

/* Copies of the loop state: G_tskij, Sigma_tskij (nt_f, ns, nk, nb, nb), Dm_skij
   (ns, nk, nb, nb); NULL entries are skipped. */
COQUI_B200_API int coqui_b200_get_scgw_state(coqui_b200_ctx* ctx, double* G_tskij,
                                             double* Sigma_tskij, double* Dm_skij);

/* Dyson equation for G from Sigma_tskij (simple_dyson::solve_dyson + Dm = -G(beta^-)); the
   result replaces the resident G.  G_tskij / Dm_skij outputs may be NULL. */
COQUI_B200_API int coqui_b200_dyson_g(coqui_b200_ctx* ctx, const double* Sigma_tskij,
                                      double* G_tskij, double* Dm_skij);

/* Galitskii-Migdal correlation energy of G_tskij and Sigma_tskij (eval_corr_energy,
   scf_common.cpp:87-136; k weights 1/nk). */
COQUI_B200_API int coqui_b200_gm_energy(coqui_b200_ctx* ctx, const double* G_tskij,
                                        const double* Sigma_tskij, double* e_corr);

/* ---- learned self-energy update: a small MLP (in -> width -> width -> out, tanh), BF16
   weights, FP32 accumulation, trained on the device by hand-written kernels.  No counterpart
   in the reference (its loop has only damping and DIIS). ---- */

COQUI_B200_API int coqui_b200_mlp_create(coqui_b200_mlp** mlp, int64_t in_dim, int64_t width,
                                         int64_t out_dim, uint64_t seed, int device);
COQUI_B200_API void coqui_b200_mlp_destroy(coqui_b200_mlp* mlp);
COQUI_B200_API const char* coqui_b200_mlp_last_error(const coqui_b200_mlp* mlp);
/* Parameters as FP32 W1 (width, in), b1, W2 (width, width), b2, W3 (out, width), b3. */
COQUI_B200_API int64_t coqui_b200_mlp_num_params(const coqui_b200_mlp* mlp);
COQUI_B200_API int coqui_b200_mlp_set_params(coqui_b200_mlp* mlp, const float* params);
COQUI_B200_API int coqui_b200_mlp_get_params(coqui_b200_mlp* mlp, float* params);
/* Y (B, out) = MLP(X (B, in)), host arrays. */
COQUI_B200_API int coqui_b200_mlp_forward(coqui_b200_mlp* mlp, const float* X, int64_t B, float* Y);
/* Mean squared error of MLP(X) against T (B, out) and its gradient (num_params). */
COQUI_B200_API int coqui_b200_mlp_gradient(coqui_b200_mlp* mlp, const float* X, const float* T,
                                           int64_t B, float* loss, float* grad);
/* Learned extrapolation (4 inputs, 2 outputs): hist (4, n) complex128, the last four iterates of
   n sequences (oldest first); with d1 = s3 - s2, d2 = s2 - s1, d3 = s1 - s0 the network maps
   (d1/d2, d2/d3) to (s_inf - s3)/d1; delta (n) complex128 = d1 * output, at most max_jump |d1|,
   0 where the differences vanish. */
COQUI_B200_API int coqui_b200_mlp_extrapolate(coqui_b200_mlp* mlp, const double* hist, int64_t n,
                                              double max_jump, double* delta);
/* Adam training over shuffled mini-batches; loss_history (epochs) may be NULL. */
COQUI_B200_API int coqui_b200_mlp_train(coqui_b200_mlp* mlp, const float* X, const float* T,
                                        int64_t n_samples, int64_t batch, int64_t epochs,
                                        double lr, uint64_t seed, float* loss_history);

/* ---- uneven batch of independent Gamma-only molecules (one k-point each, their own nb and Np,
   shared IR grid) with fused launches: grouped tensor-core GEMMs, one grouped FP64
   factorisation launch, Hadamard products and IR transforms over all molecules' columns.
   No counterpart in the reference, which runs one system per process; the per-molecule path
   is the single-system context above with nk = 1.  Mixed precision only. ---- */
typedef struct coqui_b200_batch coqui_b200_batch;

COQUI_B200_API int coqui_b200_batch_create(coqui_b200_batch** batch, int64_t nmol,
                                           const int64_t* nb, const int64_t* Np, int64_t nt_f,
                                           int64_t nw_b, int device);
COQUI_B200_API void coqui_b200_batch_destroy(coqui_b200_batch* batch);
COQUI_B200_API const char* coqui_b200_batch_last_error(const coqui_b200_batch* batch);
/* Device time (CUDA events on the batch's stream) of the last batch GW iteration, ms. */
COQUI_B200_API double coqui_b200_batch_last_ms(const coqui_b200_batch* batch);
/* Shared bosonic IR tables as for coqui_b200_set_ir (Twt_bb (nw_b, nt_f), Ttw_bb (nt_f, nw_b),
   tau_mesh_x (nt_f)). */
COQUI_B200_API int coqui_b200_batch_set_ir(coqui_b200_batch* batch, const double* Twt_bb,
                                           const double* Ttw_bb, const double* tau_mesh_x);
/* THC data of molecule m: X_Pa (Np, nb), V_PQ (Np, Np) complex128. */
COQUI_B200_API int coqui_b200_batch_set_thc(coqui_b200_batch* batch, int64_t m, const double* X_Pa,
                                            const double* V_PQ);
/* One GW iteration (update_w + evaluate) of every molecule: G_list[m] (nt_f, nb_m, nb_m) in,
   Sigma_list[m] (nt_f, nb_m, nb_m) out (the list or entries may be NULL). */
COQUI_B200_API int coqui_b200_batch_gw_iteration(coqui_b200_batch* batch,
                                                 const double* const* G_list,
                                                 double* const* Sigma_list);

/* Building blocks (same layouts as the reference's arguments). */
COQUI_B200_API int coqui_b200_primary_to_aux(coqui_b200_ctx* ctx, int64_t n_tau, const double* O_tskab,
                              double* O_tskPQ);
COQUI_B200_API int coqui_b200_aux_to_primary(coqui_b200_ctx* ctx, int64_t n_tau, const double* O_tskPQ,
                              double* O_tskab);
COQUI_B200_API int coqui_b200_tau_to_w(coqui_b200_ctx* ctx, const double* X_tqPQ, double* X_wqPQ);
COQUI_B200_API int coqui_b200_w_to_tau(coqui_b200_ctx* ctx, const double* X_wqPQ, double* X_tqPQ);
COQUI_B200_API int coqui_b200_dyson_w(coqui_b200_ctx* ctx, const double* Pi_wqPQ, double* W_wqPQ);

/* Device-timed breakdown of the last call: fills up to n (name, ms) pairs, returns count. */
COQUI_B200_API int coqui_b200_last_timings(const coqui_b200_ctx* ctx, char* names, int name_len, double* ms,
                            int n);

/* Device memory of the projected-G cache that carries G_PQ(tau) from the polarizability to
   the self-energy of the same G: -1 (default) at most half the free memory at its first use,
   0 none, else at most `bytes` (and half the free memory).  Slices outside the cache are
   projected again for the self-energy; results are the same.  Releases the current cache. */
COQUI_B200_API int coqui_b200_set_gcache_limit(coqui_b200_ctx* ctx, int64_t bytes);

/* Per-kernel CUDA-event timing (recorded on the context's stream around every launch
   group) while profiling is on; set_profiling resets the accumulators. */
COQUI_B200_API int coqui_b200_set_profiling(coqui_b200_ctx* ctx, int on);
COQUI_B200_API int coqui_b200_kernel_stats(const coqui_b200_ctx* ctx, char* names, int name_len,
                                           double* ms, int64_t* launches, int n);
/* Work units of the same groups, in the same order: the (tau, k) problems of the primary <->
   auxiliary projections ("proj_p2a", "proj_a2p"; a G(tau) projected again for the self-energy
   counts again), 0 for groups that do not count theirs. */
COQUI_B200_API int coqui_b200_kernel_units(const coqui_b200_ctx* ctx, char* names, int name_len,
                                           int64_t* units, int n);

/* Tile-shape autotuner of the tensor-core GEMMs (process-wide, on by default; the environment
   variable COQUI_B200_AUTOTUNE=0 starts with it off): the first product of each shape class
   runs every tile configuration once and keeps the fastest (all configurations give identical
   results).  coqui_b200_tuned_shapes returns the number of tuned classes. */
COQUI_B200_API void coqui_b200_set_autotune(int on);
COQUI_B200_API int64_t coqui_b200_tuned_shapes(void);

/* Pins every tensor-core GEMM to one tile configuration (0 .. coqui_b200_num_tile_configs()-1;
   -1 returns to the autotuner or heuristic), process-wide, for reproducible timing and for
   checking that the configurations agree.  Returns COQUI_B200_EINVAL for other values. */
COQUI_B200_API int coqui_b200_set_tile_config(int cfg);
COQUI_B200_API int coqui_b200_num_tile_configs(void);

/* The FP64 factorisation step of coqui_b200_dyson_w on caller-owned device buffers (from
   scr_coulomb_t::dyson_W_in_place, scr_coulomb_t.cpp:171-199, and the log-determinant of
   thc_rpa.icc:130-165, in the Hermitian form M = L^H Pi L, I - M = C C^H): for each of nprob
   Np x Np problems, M_dev complex64 (lower triangle read), A_dev complex128 workspace with
   C (lower, off the diagonal blocks) and C^{-H} inside the 128-column diagonal groups (upper)
   on return, logdet_dev[p] = 2 sum ln C_ii, trace_dev[p] (re, im) = sum M_ii, info_dev[p] = 1
   for a non-positive pivot.  Runs on `stream` (a cudaStream_t, NULL = default stream) and
   returns after it finished; allocates nothing. */
COQUI_B200_API int coqui_b200_factor_dielectric(const float* M_dev, double* A_dev,
                                                double* logdet_dev, double* trace_dev,
                                                int* info_dev, int64_t Np, int64_t nprob,
                                                void* stream);

/* Quasiparticle equation per element I < nel (solve_qp_eqn, src/methods/SCF/
   qp_scf_common.cpp:150-311): the diagonal self-energy Sigma_I(i w_n) given at nfit fermionic
   Matsubara frequencies w_fit[n] (real w_n of i w_n; sigma_fit complex128 (nfit, nel)) is
   continued to the real axis by Thiele's nfit-point Pade approximant (analyt_cont::pade_t,
   src/numerics/ac/pade/pade_t.hpp; double-double arithmetic here) and
   E_I = vhf[I] + Re Sigma_I(E_I - mu + i eta) is solved from e0[I] with method 0 "sc"
   (bisection, qp_eqn_bisection), 1 "sc_newton" (secant, qp_eqn_secant), 2 "linearized"
   (qp_eqn_linearized) or 3 "spectral" (qp_eqn_spectral), tolerance tol.  Host arrays;
   e_out, res_out (the residual at E) and conv_out (1 = converged) are written.  2 <= nfit
   <= 64.  A message goes to errbuf (may be NULL) on an error. */
COQUI_B200_API int coqui_b200_qp_solve(const double* w_fit, const double* sigma_fit,
                                       const double* vhf, const double* e0, int64_t nel, int nfit,
                                       double mu, double eta, double tol, int method, int device,
                                       double* e_out, double* res_out, int* conv_out, char* errbuf,
                                       int errlen);

/* Time limit (ns) of the bounded device-side waits of the tensor-core kernels on `device`
   (ns <= 0 restores the default of 2 s).  A kernel whose wait runs out sets an error flag,
   lets its issued tensor-core work retire, frees its tensor memory and returns; the call
   that launched it returns COQUI_B200_ETIMEDOUT and the context stays usable.  A test hook
   for that path (a limit of a few ns makes the waits run out); no reference counterpart. */
COQUI_B200_API int coqui_b200_set_wait_limit_ns(int device, int64_t ns);

/* Number of kernels this library launched since the context was created. */
COQUI_B200_API int64_t coqui_b200_kernel_launches(const coqui_b200_ctx* ctx);

/* Allocation-free primary -> auxiliary projection O^k_PQ = X^k G^k X^k^H for callers that
   own their device buffers but must not allocate device memory (an application with its
   own memory pool or a fixed device-memory budget, or code that cannot afford the device
   synchronisation cudaMalloc/cudaFree imply).  It has no counterpart in the reference: it is
   an extra entry into the same tensor-core projection that coqui_b200_primary_to_aux runs.
   X_skPa: device complex128 (nk, Np, nb); O_skab: device complex128 (nk, nb, nb);
   O_skPQ: device complex64 (nk, Np, Np), written.  Runs on `stream` (a cudaStream_t, NULL =
   default stream) and returns after the work finished.  All intermediates live in one
   static 32 MiB device array: larger problems are rejected with COQUI_B200_EINVAL and a
   message in errbuf (may be NULL).  Every device that loads the library keeps that array
   until exit; calls share it, so calls that overlap on the GPU race.  The first call on a
   device looks up the array's address; make it before any stream capture. */
COQUI_B200_API int coqui_b200_primary_to_aux_noalloc(const double* X_skPa, const double* O_skab,
                                                     float* O_skPQ, int64_t nk, int64_t Np,
                                                     int64_t nb, void* stream, char* errbuf,
                                                     int errlen);

#ifdef __cplusplus
}
#endif
#endif /* COQUI_B200_H */
