"""FP64 CPU oracle for the symmetry-reduced (IBZ) k-space paths -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy complex128, CoQui's k-space polarizability and self-energy for a mean field
with space-group and time-reversal symmetry, and the construction of the k-point lists and
maps those paths read.  Only tests, the smoke check and the benchmark's CPU legs may import it.

* ``build_bz_symmetry``: the 1st-BZ k list from the IBZ (src/mean_field/symmetry/
  bz_symmetry.hpp:48-260: IBZ points first, time-reversal partners appended, then the images of
  the operation that adds the most new points, time-reversal points moved to the end,
  ``kp_trev_pair``), the q maps of a Gamma-centred grid (:295-333, Qpts = kpts,
  qp_to_ibz = kp_to_ibz) and ``generate_qsymm_maps`` (src/utilities/symmetry.hpp:498-590);
* ``primary_to_aux_ibz``: thc_solver_comm.hpp:405-428 with kp_map / kp_trev (the IBZ matrix,
  transposed for a time-reversal image);
* ``eval_Pi_rpa_kspace``: src/methods/scr_coulomb/rpa_pi.icc:182-336;
* ``eval_Sigma_all_kspace``: src/methods/GW/thc_gw.icc:216-443 (both tau halves,
  thc_gw.cpp:170-172);
* ``update_w_kspace`` / ``rpa_energy_kspace``: scr_coulomb_t.cpp:37-95 and
  thc_rpa.icc:130-173 over the IBZ q-points with q weights;
* ``eps_inv_head_kspace`` / ``sigma_div_correction_kspace``: eps_inv_head_t over Qpts_ibz
  (g0_div_utils.hpp:55-111, 180-214) and Sigma_div_correction on the IBZ k-points
  (thc_gw.icc:446-526).

Operations act on integer crystal coordinates of the k grid: ``ops[is]`` is the integer
matrix that generates the images of the IBZ (the reference's R^-1 transposed); index 0 is the
identity.  Arrays are in the reference's own k order (IBZ first); X is (ns, nk, Np, nb) and V
(nq, Np, Np) in that order.

Parity pin: for inputs with the symmetry (built by the tests), every function here is checked
against the full-BZ R-space restatement of ``thc_oracle`` at the IBZ points.
"""
from __future__ import annotations

import numpy as np

from oracle import thc_oracle as O


def _key(m, grid):
    return tuple(int(v) % int(g) for v, g in zip(m, grid))


def build_bz_symmetry(kp_grid, ops, use_trev):
    """k list and symmetry maps of a Gamma-centred grid (bz_symmetry.hpp:48-333 with
    symmetry.hpp:498-590).  Returns a dict with integer crystal coordinates ``kc`` (nk, 3) in
    the reference's order and the maps ``kp_to_ibz``, ``kp_symm``, ``kp_trev``,
    ``kp_trev_pair``, ``qp_to_ibz``, ``qp_trev``, ``qsymms``, ``nq_per_s``, ``Qs``,
    ``ks_to_k``, ``qk_to_k2``, ``qminus``, ``nk_ibz``, ``nq_ibz``."""
    grid = tuple(int(g) for g in kp_grid)
    ops = [np.asarray(M, np.int64) for M in ops]
    nsymm = len(ops)
    allk = [(a, b, c) for a in range(grid[0]) for b in range(grid[1]) for c in range(grid[2])]

    def act(M, k):
        return _key(M @ np.asarray(k), grid)

    def neg(k):
        return _key(-np.asarray(k), grid)

    # IBZ: the first grid point (lexicographic) of every orbit under the operations (and -1)
    seen, ibz = set(), []
    for k in allk:
        if k in seen:
            continue
        ibz.append(k)
        orb = {act(M, k) for M in ops}
        if use_trev:
            orb |= {neg(x) for x in orb}
        seen |= orb
    nk_ibz = len(ibz)
    kplist = list(ibz)
    kp_s = [0] * nk_ibz
    kp_ibz = list(range(nk_ibz))
    trev = [False] * nk_ibz
    k_gamma = ibz.index((0, 0, 0))
    if nsymm > 1 or use_trev:
        if use_trev:
            for j in range(nk_ibz):
                if j == k_gamma:
                    continue
                kp = neg(kplist[j])
                if kp not in kplist:
                    kplist.append(kp)
                    kp_s.append(0)
                    kp_ibz.append(j)
                    trev.append(True)
        done = [False] * nsymm
        done[0] = True
        while True:
            best = None
            for s in range(nsymm):
                if done[s]:
                    continue
                v, idx, tf = [], [], []
                for j in range(nk_ibz):
                    if j == k_gamma:
                        continue
                    kp = act(ops[s], kplist[j])
                    if kp not in kplist and kp not in v:
                        v.append(kp)
                        idx.append(j)
                        tf.append(False)
                    if use_trev:
                        kp = neg(kp)
                        if kp not in kplist and kp not in v:
                            v.append(kp)
                            idx.append(j)
                            tf.append(True)
                if v and (best is None or len(v) > len(best[1])):
                    best = (s, v, idx, tf)
            if best is None:
                break
            s, v, idx, tf = best
            done[s] = True
            kplist += v
            kp_s += [s] * len(v)
            kp_ibz += idx
            trev += tf
    nk = len(kplist)
    if nk != len(allk):
        raise ValueError("the operations do not generate the whole grid")
    # time-reversal points to the end (order kept within both groups)
    order = [i for i in range(nk) if not trev[i]] + [i for i in range(nk) if trev[i]]
    kplist = [kplist[i] for i in order]
    kp_s = np.array([kp_s[i] for i in order], np.int64)
    kp_ibz = np.array([kp_ibz[i] for i in order], np.int64)
    trev = np.array([trev[i] for i in order], bool)
    ntrev = int(trev.sum())
    pair = np.full(nk, -1, np.int64)
    for ik in range(nk - ntrev, nk):
        for n in range(nk - ntrev):
            if kp_s[n] == kp_s[ik] and kp_ibz[n] == kp_ibz[ik]:
                if neg(kplist[ik]) != kplist[n]:
                    raise ValueError("time-reversal pair is not -k")
                pair[ik], pair[n] = n, ik
                break
        if pair[ik] < 0:
            raise ValueError("time-reversal partner not found")
    kc = np.array(kplist, np.int64)
    index = {k: i for i, k in enumerate(kplist)}
    # Gamma-centred q grid: Qpts = kpts, the q IBZ is the k IBZ (bz_symmetry.hpp:306-317)
    if nsymm == 1 and not use_trev:
        qp_symm, qp_trev, qp_to_ibz, nq_ibz = np.zeros(nk, np.int64), np.zeros(nk, bool), \
            np.arange(nk), nk
    else:
        qp_symm, qp_trev, qp_to_ibz, nq_ibz = kp_s.copy(), trev.copy(), kp_ibz.copy(), nk_ibz
    # generate_qsymm_maps (symmetry.hpp:498-590)
    unique = []
    for s in qp_symm:
        if s not in unique:
            unique.append(int(s))
    if len(unique) == 1 and unique[0] == 0 and not use_trev:
        qsymms = np.array([0])
        nq_per_s = np.array([nk])
        ks_to_k = np.arange(nk)[None, :].copy()
        Qs = np.zeros((1, 2 * nq_ibz), np.int64)
        Qs[0, :nq_ibz] = np.arange(nq_ibz)
    else:
        qsymms = np.array(unique, np.int64)
        nq_per_s = np.array([int((qp_symm == s).sum()) for s in unique], np.int64)
        ks_to_k = np.zeros((len(unique), nk), np.int64)
        Qs = np.zeros((len(unique), 2 * nq_ibz), np.int64)
        for i, s in enumerate(unique):
            js = [j for j in range(nk) if qp_symm[j] == s]
            Qs[i, :len(js)] = js
            Rt = np.rint(np.linalg.inv(ops[s])).astype(np.int64)  # R^T = (R^-1 T)^-1
            for ik in range(nk):
                ks_to_k[i, ik] = index[act(Rt, kplist[ik])]
    qk_to_k2 = np.array([[index[_key(np.asarray(kplist[k]) - np.asarray(kplist[q]), grid)]
                          for k in range(nk)] for q in range(nk)], np.int64)
    qminus = np.array([index[neg(kplist[q])] for q in range(nk)], np.int64)
    lex = np.array([(k[0] * grid[1] + k[1]) * grid[2] + k[2] for k in kplist], np.int64)
    return dict(kc=kc, lex=lex, nk=nk, nk_ibz=nk_ibz, nq_ibz=nq_ibz, kp_to_ibz=kp_ibz,
                kp_symm=kp_s, kp_trev=trev, kp_trev_pair=pair, qp_to_ibz=qp_to_ibz,
                qp_symm=qp_symm, qp_trev=qp_trev, qsymms=qsymms, nq_per_s=nq_per_s, Qs=Qs,
                ks_to_k=ks_to_k, qk_to_k2=qk_to_k2, qminus=qminus, grid=grid)


def primary_to_aux_ibz(O_ibz, X_skPa, kp_to_ibz, kp_trev, nk=None):
    """thc_solver_comm.hpp:405-428: O^k_PQ = X^k_Pa O^{kp_map(k)}_ab conj(X^k_Qb), with the
    IBZ matrix transposed when kp_trev(k).  O_ibz (..., ns, nk_ibz, nb, nb) ->
    (..., ns, nk, Np, Np) for the first nk k-points (all by default)."""
    nk = X_skPa.shape[1] if nk is None else nk
    Ok = O_ibz[..., np.asarray(kp_to_ibz[:nk]), :, :]
    tr = np.asarray(kp_trev[:nk], bool)
    Ok = np.where(tr[:, None, None], np.swapaxes(Ok, -1, -2), Ok)
    return O.primary_to_aux(Ok, X_skPa[:, :nk])


def eval_Pi_rpa_kspace(G_tskij, X_skPa, sym) -> np.ndarray:
    """rpa_pi.icc:182-336: Pi_q = factor sum_k conj(G_PQ^{k-q}(t)) G_PQ^k(beta - t) for the
    IBZ q-points, factor = -2/nk (ns = 1) or -1/nk; (nt_half, nq_ibz, Np, Np)."""
    nt, ns, _, nb, _ = G_tskij.shape
    nk = X_skPa.shape[1]
    Np = X_skPa.shape[2]
    nt_half = (nt + 1) // 2
    factor = (-1.0 if ns == 2 else -2.0) / nk
    nq_ibz = sym["nq_ibz"]
    k2 = sym["qk_to_k2"]
    Pi = np.zeros((nt_half, nq_ibz, Np, Np), np.complex128)
    for it in range(nt_half):
        Gp = np.conj(primary_to_aux_ibz(G_tskij[it], X_skPa, sym["kp_to_ibz"], sym["kp_trev"]))
        Gn = primary_to_aux_ibz(G_tskij[nt - it - 1], X_skPa, sym["kp_to_ibz"], sym["kp_trev"])
        for iq in range(nq_ibz):
            for s in range(ns):
                for ik in range(nk):
                    Pi[it, iq] += factor * (Gp[s, k2[iq, ik]] * Gn[s, ik])
    return Pi


def eval_Sigma_all_kspace(G_tskij, dW_qtPQ, X_skPa, sym, D=None) -> np.ndarray:
    """thc_gw.icc:216-443, called for t and for beta - t (thc_gw.cpp:170-172).  G_tskij is
    on the IBZ k-points, dW_qtPQ (nq_ibz, nt_half, Np, Np); D (nsym, nk_ibz, nb, nb) are the
    rotations d[isym, k] (row 0 unused).  Returns Sigma (nt, ns, nk_ibz, nb, nb)."""
    nt, ns, nk_ibz, nb, _ = G_tskij.shape
    nk = X_skPa.shape[1]
    nt_half = (nt + 1) // 2
    factor = -1.0 / nk
    ntrev = int(np.asarray(sym["kp_trev"]).sum())
    nk_nt = nk - ntrev
    kp_trev, pair = sym["kp_trev"], sym["kp_trev_pair"]
    qp_trev, qminus, k2 = sym["qp_trev"], sym["qminus"], sym["qk_to_k2"]
    Sigma = np.zeros((nt, ns, nk_ibz, nb, nb), np.complex128)
    for minus_t in (False, True):
        for it in range(nt_half):
            itg = nt - it - 1 if minus_t else it
            Gaux = primary_to_aux_ibz(G_tskij[itg], X_skPa, sym["kp_to_ibz"], kp_trev, nk_nt)
            for i, _ in enumerate(sym["qsymms"]):
                S = np.zeros((ns, nk_ibz) + Gaux.shape[-2:], np.complex128)
                for s in range(ns):
                    for ik in range(nk_ibz):
                        ks = sym["ks_to_k"][i, ik]
                        for j in range(sym["nq_per_s"][i]):
                            qp = sym["Qs"][i, j]
                            qs = sym["qp_to_ibz"][qp]
                            W = dW_qtPQ[qs, it]
                            if qp_trev[qp]:
                                km = k2[qminus[qs], ks]
                                if kp_trev[km]:
                                    S[s, ik] += np.conj(factor * (W * Gaux[s, pair[km]]))
                                else:
                                    S[s, ik] += factor * (Gaux[s, km] * np.conj(W))
                            else:
                                km = k2[qs, ks]
                                if kp_trev[km]:
                                    S[s, ik] += factor * (W * np.conj(Gaux[s, pair[km]]))
                                else:
                                    S[s, ik] += factor * (Gaux[s, km] * W)
                # aux_to_primary with X at ks_to_k(isym, k)
                Xs = X_skPa[:, sym["ks_to_k"][i, :nk_ibz]]
                Sab = O.aux_to_primary(S, Xs)
                if minus_t and itg == nt_half - 1:
                    continue  # thc_gw.icc:297-298 (odd nt: the middle slice counted once)
                if i == 0:
                    Sigma[itg] += Sab
                else:
                    Dk = D[i]  # (nk_ibz, nb, nb)
                    Sigma[itg] += np.conj(np.swapaxes(Dk, -1, -2))[None] @ Sab @ Dk[None]
    return Sigma


def q_weights(sym) -> np.ndarray:
    """thc_rpa.icc:133: the number of 1st-BZ q-points that map to each IBZ q-point."""
    return np.bincount(np.asarray(sym["qp_to_ibz"]), minlength=sym["nq_ibz"]).astype(np.float64)


def update_w_kspace(G_tskij, X_skPa, V_qPQ, ft, sym):
    """scr_coulomb_t.cpp:37-95 over the IBZ q-points: Pi -> tau_to_w -> Dyson with V of the
    IBZ q-points -> w_to_tau; returns dW_qtPQ (nq_ibz, nt_half, Np, Np)."""
    Pi_t = eval_Pi_rpa_kspace(G_tskij, X_skPa, sym)
    Pi_w = ft.tau_to_w_PHsym(Pi_t)
    W_w = O.dyson_W_in_place(Pi_w, V_qPQ[:sym["nq_ibz"]])
    W_t = ft.w_to_tau_PHsym(W_w)
    return np.ascontiguousarray(np.swapaxes(W_t, 0, 1))


def rpa_energy_kspace(G_tskij, X_skPa, V_qPQ, ft, sym) -> float:
    """thc_rpa.icc:21-181 with the IBZ q-points weighted by their multiplicity."""
    Pi_t = eval_Pi_rpa_kspace(G_tskij, X_skPa, sym)
    Pi_w = ft.tau_to_w_PHsym(Pi_t)
    return O.rpa_energy_from_Pi_w(Pi_w, V_qPQ[:sym["nq_ibz"]], ft, X_skPa.shape[1],
                                  q_weight=q_weights(sym))


def eps_inv_head_kspace(dW_qtPQ, chi_bar_qP, Qpts_ibz, lattv, ft, div="ignore_g0"):
    """eps_inv_head_t on the IBZ q-points: eps^-1(t, q) of W(q_ibz) with the chi-bar heads of
    those q-points, then the head of the treatment (g0_div_utils.hpp:55-111, 180-214)."""
    W_tq = np.swapaxes(dW_qtPQ, 0, 1)
    eps = O.eval_eps_inv_q(W_tq, chi_bar_qP, Qpts_ibz, lattv)
    return O.eps_inv_head_t(eps, Qpts_ibz, ft, div)


def sigma_div_correction_kspace(Sigma_tskij, G_tskij, X_skPa, chi_head_P, eps_inv_head,
                                madelung, div, nq_ibz):
    """Sigma_div_correction (thc_gw.icc:446-526) on the IBZ k-points: X of the first nk_ibz
    k-points (the IBZ), nothing when nqpts_ibz == 1."""
    nk_ibz = G_tskij.shape[2]
    return O.sigma_div_correction(Sigma_tskij, G_tskij, X_skPa[:, :nk_ibz], chi_head_P,
                                  eps_inv_head, madelung, div, nq=nq_ibz)
