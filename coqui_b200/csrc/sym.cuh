// Kernels of the symmetry-reduced (IBZ) k-space path (sym.cu).
//
// The reference's k-space forms (rpa_pi.icc:182-336, thc_gw.icc:216-443) read the Green's
// function on the IBZ k-points only and produce the screened interaction on the IBZ q-points;
// the self-energy of each IBZ k-point is a sum over the 1st-BZ q-points, split by the
// symmetry operation that maps each q-point into the IBZ.
#pragma once

#include "common.cuh"

namespace cq {

// G (nt, nk, nb, nb) complex128 in lexicographic k order from the IBZ matrices
// Gi (nt, nk_ibz, nb, nb): G[t, k] = Gi[t, src[k] & 0x3fffffff], transposed when bit 30 of
// src[k] is set (the time-reversal image, thc_solver_comm.hpp:421-425).
void launch_unfold_g(const double2* Gi, double2* G, const int* src, int64_t nt, int64_t nk,
                     int64_t nk_ibz, int64_t nb, cudaStream_t s);

// out[t, i] = transpose(in[t, qsrc[i]]) for i < nqo: (nt, nq, Np, Np) -> (nt, nqo, Np, Np) in
// storage precision R (the k-space polarizability of an IBZ q-point is the transposed R-space
// one of -q).
template <typename R>
void launch_gather_transpose(const cplx_t<R>* in, cplx_t<R>* out, const int* qsrc, int64_t nt,
                             int64_t nq, int64_t nqo, int64_t Np, cudaStream_t s);

// Self-energy rows of one tau slice: row p = (isym, ik) is the sum of its terms (w, g, flags),
// each factor * (flags & 1 ? conj(G[g]) : G[g]) * (flags & 2 ? conj(W[w]) : W[w]) element-wise;
// rows[p] = (first term, term count).  G (nk, ncol) and W (nqi, ncol) in storage precision R,
// S (nrow, ncol); accumulation in the storage precision.  Every G and W column tile is read
// from HBM once.
template <typename R>
void launch_sigma_ksum(const cplx_t<R>* G, const cplx_t<R>* W, const int4* terms,
                       const int2* rows, int64_t nrow, int64_t nk, int64_t nqi, int64_t ncol,
                       double factor, cplx_t<R>* S, cudaStream_t s);

// out[i] += sum over b < nblk of Rb[b * n + i] (complex128)
void launch_add_blocks(const double2* Rb, double2* out, int64_t nblk, int64_t n, cudaStream_t s);

}  // namespace cq
