// Device pieces of the self-consistent GW loop (nb x nb sized work): Dyson equation for G on
// the fermionic Matsubara grid, Hermitian symmetrisation, trace products for the energies,
// damping and the commutator-DIIS vector algebra.
#pragma once

#include <complex>
#include <vector>

#include "common.cuh"

namespace cq {

// A <- (A + A^H) / 2 for nmat consecutive nb x nb complex128 matrices
void hermitize_c128(double2* A, int64_t nb, int64_t nmat, cudaStream_t s);

// out[m] = sum_ij A[m]_ij B[bm]_ji with bm = m % b_mod (b_mod = 0: bm = m)
void trace_products(const double2* A, const double2* B, double2* out, int64_t nb, int64_t nmat,
                    int64_t b_mod, cudaStream_t s);

// X[w, k] = (i pi wn[w] / beta + mu) S[k] - H0[k] - F[k] - Sigma[w, k] for nw x nk matrices
void build_dyson_matrix(const double2* S, const double2* H0, const double2* F,
                        const double2* Sigma_w, double2* X, const int64_t* wn, double beta,
                        double mu, int64_t nw, int64_t nk, int64_t nb, cudaStream_t s);

// In-place FP64 inverse of nmat nb x nb complex matrices (Gauss-Jordan with partial pivoting,
// one CTA per matrix, the matrix in shared memory; nb <= 96).  info[m] = 1 marks a singular
// matrix.
void invert_batched(double2* A, int64_t nb, int64_t nmat, int* info, cudaStream_t s);

// y = a x + b y (real a, b), n complex values
void axpby_c128(const double2* x, double2* y, double a, double b, int64_t n, cudaStream_t s);
// y += c x (complex c)
void axpy_c128(const double2* x, double2* y, double2 c, int64_t n, cudaStream_t s);

// Reductions (host result, synchronous on s): max_i |a_i - b_i| (b may be null: max |a_i|)
// and sum_i conj(a_i) b_i.
double maxabs_diff(const double2* a, const double2* b, int64_t n, DevBuf<double>& part,
                   cudaStream_t s);
std::complex<double> dotc(const double2* a, const double2* b, int64_t n, DevBuf<double>& part,
                          cudaStream_t s);

// out[m * nb + i] = A[m]_ii, and A[m]_ii += d[m * nb + i], for nmat nb x nb matrices
void extract_diag(const double2* A, double2* out, int64_t nb, int64_t nmat, cudaStream_t s);
void add_diag(double2* A, const double2* d, int64_t nb, int64_t nmat, cudaStream_t s);

// Hartree pieces of THC Hartree-Fock (FP64): rho[Q] = scale sum_k sum_b T[k,Q,b] conj(X[k,Q,b])
// for T = X Dm per k (the diagonal of X Dm X^H summed over k), and Y[k,P,b] = d[P] X[k,P,b].
void aux_diag(const double2* T, const double2* X, double2* rho, int64_t nk, int64_t Np,
              int64_t nb, double scale, cudaStream_t s);
void scale_rows(const double2* X, const double2* d, double2* Y, int64_t nk, int64_t Np,
                int64_t nb, cudaStream_t s);

// A[s * per + e] *= f[s] (real f) for nslice consecutive slices of per complex values
void scale_slices(double2* A, const double* f, int64_t nslice, int64_t per, cudaStream_t s);

// Eigen-decomposition of a small real symmetric matrix by cyclic Jacobi rotations (host):
// A (n x n, row-major) -> ev (n), U (n x n, row-major, column k = eigenvector k).
void sym_eigen(const std::vector<double>& A, int64_t n, std::vector<double>& ev,
               std::vector<double>& U);

}  // namespace cq
