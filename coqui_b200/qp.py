"""Quasiparticle GW loops (G0W0 and eigenvalue-self-consistent evGW) on the device path.

Mirrors CoQui's ``qp_scf_loop<evscf_only = true>`` (src/methods/SCF/scf_driver.cpp:190-353)
with ``add_evscf_vcorr`` (src/methods/SCF/qp_scf_common.cpp:313-378): per iteration

1. with Hartree-Fock on, H_eff = H0 + J + K of the current density matrix
   (``coqui_b200_hf_evaluate``, as ``hf_t::evaluate`` plus H0 in the loop);
2. G(tau) from the fixed molecular orbitals C and the current energies E (``update_G``,
   qp_scf_common.cpp:82-118), then W and Sigma(tau) of that G on the GPU
   (``coqui_b200_gw_iteration``: update_w + gw_t::evaluate);
3. ``solve_qp_eqn`` (:150-311): diag(C^H Sigma(tau) C) brought to the fermionic Matsubara
   axis, V_hf = diag(C^H H_eff C), and E = V_hf + Re Sigma(E - mu + i eta) solved on the GPU
   from an N-point Pade continuation (``coqui_b200_qp_solve``);
4. H_eff = C^{-H} diag(E) C^{-1}, the change of H_eff as the convergence measure
   (``solve_iterative`` with plain mixing), then mu (``update_mu``) and the density matrix.

With Hartree-Fock off H_eff carries over between iterations exactly as in the reference
(there the HF solver is what resets it), so one iteration is the one-shot G0W0
quasiparticle energy of the mean field.  Host work here is small (nb-sized matrices, the
MO projection of the diagonal of Sigma); the GW step and the continuation run on the GPU.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import capi


@dataclass
class QPContext:
    """qp_context_t (src/methods/SCF/qp_context.h): equation, Pade points, broadening, tolerance."""
    qp_type: str = "sc"
    Nfit: int = 18
    eta: float = 1e-4
    tol: float = 1e-8


def fit_indices(niw_pos: int, nfit: int):
    """Indices into the positive half of the fermionic mesh of the Pade fit points: evenly
    spaced, with the remainder taken by a denser low-frequency part (pade_driver.hpp:40-62)."""
    if nfit > niw_pos:
        raise ValueError(f"Nfit ({nfit}) > positive Matsubara frequencies ({niw_pos})")
    lchunk = niw_pos % nfit
    if lchunk:
        step = niw_pos // nfit + 1
        idx = list(range(0, step * lchunk, step)) + list(range(step * lchunk, niw_pos, step - 1))
    else:
        idx = list(range(0, niw_pos, niw_pos // nfit))
    if len(idx) != nfit:
        raise ValueError("fit_indices: inconsistent point count")
    return idx


def greens_function(MO_skia, E_ska, mu, ft):
    """G_tskij = sum_a C_ia g(E_a, tau) conj(C_ja), g = -e^{-(E-mu) tau} / (1 + e^{-(E-mu) beta})
    written without overflow on either side of mu (qp_scf_common.cpp:82-118)."""
    tau = ft.tau_mesh()[:, None, None, None]
    x = (np.asarray(E_ska).real - mu)[None]
    pos = x > 0
    xp, xn = np.where(pos, x, 0.0), np.where(pos, 0.0, x)
    g = np.where(pos, -np.exp(-xp * tau) / (1.0 + np.exp(-xp * ft.beta)),
                 -np.exp(xn * (ft.beta - tau)) / (1.0 + np.exp(xn * ft.beta)))
    return np.einsum("skia,tska,skja->tskij", MO_skia, g, np.conj(MO_skia))


def density_matrix(MO_skia, E_ska, mu, beta):
    """Dm_ij = sum_a C_ia f(E_a) conj(C_ja) with Fermi-Dirac occupations."""
    x = (np.asarray(E_ska).real - mu) * beta
    f = 0.5 * (1.0 - np.tanh(0.5 * x))
    return np.einsum("skia,ska,skja->skij", MO_skia, f, np.conj(MO_skia))


def compute_nelec(mu, E_ska, beta, k_weight):
    """Electrons per cell of the energies E at chemical potential mu (qp_scf_common.cpp:727-748)."""
    x = (np.asarray(E_ska).real - mu) * beta
    f = 0.5 * (1.0 - np.tanh(0.5 * x))
    nel = float(np.sum(np.asarray(k_weight)[None, :, None] * f))
    return 2.0 * nel if np.asarray(E_ska).shape[0] == 1 else nel


def update_mu(old_mu, nel_target, E_ska, beta, k_weight, mu_tol=1e-9):
    """Bisection for the chemical potential (qp_scf_common.cpp:750-803)."""
    nel = compute_nelec(old_mu, E_ska, beta, k_weight)
    if abs(nel - nel_target) < mu_tol:
        return old_mu
    delta = 0.2
    if nel >= nel_target:
        mu2, mu1 = old_mu, old_mu - delta
        while compute_nelec(mu1, E_ska, beta, k_weight) > nel_target:
            mu1 -= delta
    else:
        mu1, mu2 = old_mu, old_mu + delta
        while compute_nelec(mu2, E_ska, beta, k_weight) < nel_target:
            mu2 += delta
    mid = 0.5 * (mu1 + mu2)
    nel = compute_nelec(mid, E_ska, beta, k_weight)
    for _ in range(200):
        if abs(nel - nel_target) < mu_tol:
            break
        if nel >= nel_target:
            mu2 = mid
        else:
            mu1 = mid
        mid = 0.5 * (mu1 + mu2)
        nel = compute_nelec(mid, E_ska, beta, k_weight)
    return mid


def sigma_mo_w(Sigma_tskij, MO_skia, ft):
    """diag(C^H Sigma(tau) C) per (s, k, a), brought to the fermionic Matsubara axis
    (qp_scf_common.cpp:180-203): (nw_f, ns, nk, nbnd) complex."""
    S = np.einsum("skia,tskij,skja->tska", np.conj(MO_skia), Sigma_tskij, MO_skia, optimize=True)
    nt = S.shape[0]
    return (ft.Twt_ff @ S.reshape(nt, -1)).reshape((ft.Twt_ff.shape[0],) + S.shape[1:])


def solve_qp_eqn(E_ska, Sigma_tskij, Vhf_skij, MO_skia, mu, ft, qp: QPContext, device=0):
    """New quasiparticle energies (ns, nk, nbnd) and the per-element convergence flags."""
    Sw = sigma_mo_w(Sigma_tskij, MO_skia, ft)
    V = np.einsum("skia,skij,skja->ska", np.conj(MO_skia), Vhf_skij, MO_skia).real
    nw = Sw.shape[0]
    idx = [nw // 2 + i for i in fit_indices(nw // 2, qp.Nfit)]
    w_fit = np.array([np.pi * float(ft.wn_mesh_f[i]) / ft.beta for i in idx])
    sig = np.ascontiguousarray(Sw[idx].reshape(len(idx), -1))
    E, _, conv = capi.qp_solve(w_fit, sig, V.reshape(-1), np.asarray(E_ska).real.reshape(-1), mu,
                               qp.eta, qp.tol, qp.qp_type, device)
    return E.reshape(V.shape), conv.reshape(V.shape)


def canonical_orbitals(Heff_skij, S_skij):
    """MO coefficients and energies: H C = S C E per (s, k) (update_MOs)."""
    from scipy.linalg import eigh
    ns, nk, nb, _ = Heff_skij.shape
    E = np.empty((ns, nk, nb))
    C = np.empty((ns, nk, nb, nb), np.complex128)
    for s in range(ns):
        for k in range(nk):
            H = 0.5 * (Heff_skij[s, k] + np.conj(Heff_skij[s, k].T))
            E[s, k], C[s, k] = eigh(H, S_skij[s, k])
    return C, E


def eval_hf_energy(Dm_skij, Heff_skij, H0_skij, k_weight):
    """e_1e = spin sum_k w_k Tr[Dm H0], e_hf = spin sum_k w_k Tr[Dm (H_eff - H0)] / 2
    (scf_common.cpp:44-77 with the H0-containing effective Hamiltonian)."""
    w = np.asarray(k_weight, np.complex128)
    spin = 1.0 if Dm_skij.shape[0] == 2 else 2.0
    e_1e = np.einsum("k,skij,skji->", w, Dm_skij, H0_skij)
    e_hf = 0.5 * np.einsum("k,skij,skji->", w, Dm_skij, Heff_skij - H0_skij)
    return float((spin * e_1e).real), float((spin * e_hf).real)


def evgw_loop(ctx, H0_skij, S_skij, Fmf_skij, ft, nelec, niter=1, conv_tol=1e-6, hf=False,
              div="ignore_g0", madelung=0.0, qp: QPContext | None = None, mixing=1.0,
              device=0):
    """Eigenvalue-self-consistent GW (one iteration: G0W0) through a configured context
    (set_ir, set_ir_fermi, set_kmesh, set_thc done).  H0, S and the mean-field Fock part F
    are (ns, nk, nb, nb); the loop starts from H_eff = H0 + F.  Returns a dict with the final
    energies, mu, and the per-iteration history (energies, convergence measure, mu)."""
    qp = qp or QPContext()
    nk = H0_skij.shape[1]
    k_weight = np.full(nk, 1.0 / nk)
    Heff = H0_skij + Fmf_skij
    C, E = canonical_orbitals(Heff, S_skij)
    mu = update_mu(0.0, nelec, E, ft.beta, k_weight)
    Dm = density_matrix(C, E, mu, ft.beta)
    Heff_mf = H_out = Heff.copy()
    Cinv = np.linalg.inv(C)
    history = []
    for it in range(1, niter + 1):
        if hf:
            Heff = ctx.hf_evaluate(Dm, S_skij, True, True, div, madelung) + H0_skij
        G = greens_function(C, E, mu, ft)
        Sigma, _ = ctx.gw_iteration(G)
        E_new, conv = solve_qp_eqn(E, Sigma, Heff, C, mu, ft, qp, device)
        H_new = np.einsum("skai,ska,skaj->skij", np.conj(Cinv), E_new, Cinv)
        # solve_iterative: against the mean field at the first iteration, else against the
        # previous iteration's output (its checkpoint), with plain mixing
        prev = Heff_mf if it == 1 else H_out
        H_new = mixing * H_new + (1.0 - mixing) * prev
        dH = float(np.abs(H_new - prev).max())
        Heff = H_out = H_new
        E = E_new
        mu = update_mu(mu, nelec, E, ft.beta, k_weight)
        Dm = density_matrix(C, E, mu, ft.beta)
        e_1e, e_hf = eval_hf_energy(Dm, Heff, H0_skij, k_weight)
        history.append(dict(iteration=it, E=E.copy(), mu=mu, dHeff=dH, e_1e=e_1e, e_hf=e_hf,
                            unconverged=int((~conv).sum())))
        if dH <= abs(conv_tol):
            break
    return dict(E=E, mu=mu, Heff=Heff, MO=C, history=history)
