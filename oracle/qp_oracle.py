"""Oracle (test infrastructure only): the quasiparticle equation of CoQui's qp-scf loops.

A plain restatement of the reference, used by the tests to check the library; nothing in the
product imports it.

* ``pade_fit`` / ``pade_eval``: Thiele's reciprocal-difference Pade approximant in 100-digit
  decimal arithmetic (``src/numerics/ac/pade/pade_t.hpp`` fit :156-169, evaluate :100-120,
  ``cpp_dec_float<100>``).
* ``fit_indices``: the Matsubara points the Pade driver fits (``pade_driver.hpp:40-62``).
* ``qp_eqn_*``: the four rules of ``solve_qp_eqn`` (``src/methods/SCF/qp_scf_common.cpp``:
  spectral :560-617, linearized :619-627, secant :629-676, bisection :678-748).
* ``sigma_mo_w``: diag(C^H Sigma(tau) C) on the fermionic Matsubara axis (:180-203).
* ``update_mu`` / ``compute_nelec``: the chemical-potential bisection (:740-803).
* ``evgw_loop``: ``qp_scf_loop<evscf_only = true>`` (``scf_driver.cpp:190-353``) with
  ``add_evscf_vcorr`` (``qp_scf_common.cpp:313-378``) on the FP64 THC oracle.

Pinning: the reference ships no quasiparticle energies for THC inputs; the Pade approximant
is pinned by known answers (a rational function with fewer poles than half the fit points
is reproduced exactly), the rest by the restatement.
"""
from __future__ import annotations

from decimal import Decimal, localcontext

import numpy as np

PREC = 100


class _C:
    """Complex number of two Decimals (arithmetic in the caller's decimal context)."""

    __slots__ = ("re", "im")

    def __init__(self, re, im):
        self.re, self.im = re, im

    @staticmethod
    def of(z):
        z = complex(z)
        return _C(Decimal(z.real), Decimal(z.imag))

    def __add__(self, o):
        return _C(self.re + o.re, self.im + o.im)

    def __sub__(self, o):
        return _C(self.re - o.re, self.im - o.im)

    def __mul__(self, o):
        return _C(self.re * o.re - self.im * o.im, self.re * o.im + self.im * o.re)

    def __truediv__(self, o):
        d = o.re * o.re + o.im * o.im
        return _C((self.re * o.re + self.im * o.im) / d, (self.im * o.re - self.re * o.im) / d)

    def to_complex(self):
        return complex(float(self.re), float(self.im))


def pade_fit(z_fit, A_fit):
    """Thiele coefficients a_i = g_i(z_i), g_0 = A, g_i(z_j) = (g_{i-1}(z_{i-1}) - g_{i-1}(z_j))
    / ((z_j - z_{i-1}) g_{i-1}(z_j)) (pade_t.hpp:156-169)."""
    with localcontext() as ctx:
        ctx.prec = PREC
        z = [_C.of(v) for v in z_fit]
        n = len(z)
        g = [_C.of(v) for v in A_fit]
        for i in range(1, n):
            gd = g[i - 1]
            for j in range(i, n):
                g[j] = (gd - g[j]) / ((z[j] - z[i - 1]) * g[j])
        return z, g


def pade_eval(fit, w):
    """a_0 / (1 + a_1 (w - z_0) / (1 + ... a_{n-1} (w - z_{n-2}))) (pade_t.hpp:100-120)."""
    z, a = fit
    n = len(a)
    with localcontext() as ctx:
        ctx.prec = PREC
        wc = _C.of(w)
        one = _C(Decimal(1), Decimal(0))
        X = a[n - 1] * (wc - z[n - 2])
        for f in range(1, n - 1):
            idx = n - f - 1
            X = a[idx] * (wc - z[idx - 1]) / (one + X)
        X = a[0] / (one + X)
        return X.to_complex()


def fit_indices(niw_pos, nfit):
    """Indices (into the positive half of the fermionic mesh) of the fit points
    (pade_driver.hpp:40-62)."""
    if nfit > niw_pos:
        raise ValueError("Nfit > number of positive frequencies")
    lchunk = niw_pos % nfit
    if lchunk:
        step = niw_pos // nfit + 1
        low = list(range(0, step * lchunk, step))
        high = list(range(step * lchunk, niw_pos, step - 1))
        idx = low + high
    else:
        idx = list(range(0, niw_pos, niw_pos // nfit))
    assert len(idx) == nfit
    return idx


def qp_eqn_linearized(vhf, sig, mu, eps_ks, eta):
    h = 1e-6
    s0 = sig(complex(eps_ks - mu, eta)).real
    ds = sig(complex(eps_ks - mu + h, eta)).real - s0
    Z = 1.0 / (1.0 - ds / h)
    return Z * (vhf + s0 - (1 - 1.0 / Z) * eps_ks)


def _res(vhf, sig, mu, e, eta):
    return (complex(e, eta) - vhf - sig(complex(e - mu, eta))).real


def qp_eqn_secant(vhf, sig, mu, w0, maxiter, tol, eta):
    eps = 1e-4
    p0 = w0
    p1 = w0 * (1 + eps) + eps if p0 >= 0 else w0 * (1 + eps) - eps
    q0, q1 = _res(vhf, sig, mu, p0, eta), _res(vhf, sig, mu, p1, eta)
    if abs(q1) < abs(q0):
        p0, p1, q0, q1 = p1, p0, q1, q0
    conv, p = False, p1
    for _ in range(maxiter):
        if abs(q1) > abs(q0):
            p = (-q0 / q1 * p1 + p0) / (1 - q0 / q1)
        else:
            p = (-q1 / q0 * p0 + p1) / (1 - q1 / q0)
        if abs(p - p1) < tol:
            conv = True
            break
        p0, q0, p1 = p1, q1, p
        q1 = _res(vhf, sig, mu, p1, eta)
    return p, _res(vhf, sig, mu, p, eta), conv


def qp_eqn_bisection(vhf, sig, mu, eps0, tol, eta):
    res = _res(vhf, sig, mu, eps0, eta)
    if abs(res) < tol:
        return eps0, res
    delta = 0.01
    if res >= 0:
        e2, e1 = eps0, eps0 - delta
        r1 = _res(vhf, sig, mu, e1, eta)
        while r1 > 0:
            e1 -= delta
            r1 = _res(vhf, sig, mu, e1, eta)
    else:
        e1, e2 = eps0, eps0 + delta
        r2 = _res(vhf, sig, mu, e2, eta)
        while r2 < 0:
            e2 += delta
            r2 = _res(vhf, sig, mu, e2, eta)
    em = 0.5 * (e1 + e2)
    res = _res(vhf, sig, mu, em, eta)
    while abs(res) > tol:
        if res >= 0:
            e2 = em
        else:
            e1 = em
        em = 0.5 * (e1 + e2)
        res = _res(vhf, sig, mu, em, eta)
    return em, res


def qp_eqn_spectral(vhf, sig, mu, eps0, tol, eta):
    nw = 1000
    wmin, wmax = eps0 - mu - 1.0, eps0 - mu + 1.0
    grid = [wmin + i * (wmax - wmin) / (nw - 1) for i in range(nw)]

    def A(x):
        w = complex(x, eta)
        return abs((1.0 / (w + mu - vhf - sig(w))).imag)
    vals = [A(x) for x in grid]
    nmax = int(np.argmax(vals))
    amax = vals[nmax]
    x = grid[nmax]
    ax = A(x + tol)
    step = tol
    if ax < amax:
        step = -tol
        ax = A(x + step)
    while ax >= amax:
        x += step
        amax = ax
        ax = A(x + step)
    return x + mu, True


def sigma_mo_w(Sigma_tskij, MO_skia, ft):
    """diag(C^H Sigma(tau) C) per (s, k, a), then tau -> i w_n (fermionic):
    (nw_f, ns, nk, nbnd)."""
    S = np.einsum("skia,tskij,skja->tska", np.conj(MO_skia), Sigma_tskij, MO_skia)
    return ft.tau_to_w(S, "fermi")


def solve_qp_eqn(E_ska, Sigma_tskij, Vhf_skij, MO_skia, mu, ft, qp_type="sc", nfit=18,
                 eta=1e-4, tol=1e-8):
    """New quasiparticle energies (ns, nk, nbnd) (qp_scf_common.cpp:150-311)."""
    Sw = sigma_mo_w(Sigma_tskij, MO_skia, ft)
    V = np.einsum("skia,skij,skja->ska", np.conj(MO_skia), Vhf_skij, MO_skia).real
    nw = Sw.shape[0]
    niw_pos = nw // 2
    idx = [nw // 2 + i for i in fit_indices(niw_pos, nfit)]
    z = [ft.omega(int(ft.wn_mesh_f[i])) for i in idx]
    out = np.empty_like(E_ska, dtype=np.float64)
    for I in np.ndindex(E_ska.shape):
        fit = pade_fit(z, [Sw[(i,) + I] for i in idx])
        sig = (lambda f: (lambda w: pade_eval(f, w)))(fit)
        e0, v = float(E_ska[I].real), float(V[I])
        if qp_type in ("sc", "sc_bisection"):
            out[I] = qp_eqn_bisection(v, sig, mu, e0, tol, eta)[0]
        elif qp_type == "sc_newton":
            out[I] = qp_eqn_secant(v, sig, mu, e0, 400, tol, eta)[0]
        elif qp_type == "linearized":
            out[I] = qp_eqn_linearized(v, sig, mu, e0, eta)
        else:
            out[I] = qp_eqn_spectral(v, sig, mu, e0, tol, eta)[0]
    return out


def compute_nelec(mu, E_ska, beta, k_weight):
    # 1 / (1 + e^x) written as (1 - tanh(x / 2)) / 2, which does not overflow
    f = 0.5 * (1.0 - np.tanh(0.5 * (E_ska.real - mu) * beta))
    nel = float(np.sum(k_weight[None, :, None] * f))
    return 2.0 * nel if E_ska.shape[0] == 1 else nel


def update_mu(old_mu, nel_target, E_ska, beta, k_weight, mu_tol=1e-9):
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
    while abs(nel - nel_target) >= mu_tol:
        if nel >= nel_target:
            mu2 = mid
        else:
            mu1 = mid
        mid = 0.5 * (mu1 + mu2)
        nel = compute_nelec(mid, E_ska, beta, k_weight)
    return mid


def _eigh(H, S):
    from scipy.linalg import eigh
    ns, nk, nb, _ = H.shape
    E = np.empty((ns, nk, nb))
    C = np.empty((ns, nk, nb, nb), np.complex128)
    for s in range(ns):
        for k in range(nk):
            E[s, k], C[s, k] = eigh(0.5 * (H[s, k] + H[s, k].conj().T), S[s, k])
    return C, E


def _dm(C, E, mu, beta):
    f = 0.5 * (1.0 - np.tanh(0.5 * (E - mu) * beta))
    return np.einsum("skia,ska,skja->skij", C, f, np.conj(C))


def evgw_loop(system, ft, nelec, niter=1, conv_tol=1e-6, hf=False, div="ignore_g0",
              madelung=0.0, qp_type="sc", nfit=18, eta=1e-4, tol=1e-8, mixing=1.0):
    """qp_scf_loop<evscf_only = true> (scf_driver.cpp:190-353) for a synthetic THC system on
    the FP64 oracle: H_eff = H0 + F_mf at the start; per iteration HF (optional), G from the
    fixed orbitals and the current energies, W and Sigma, the quasiparticle equation,
    H_eff = C^{-H} diag(E) C^{-1}, mixing, mu and the density matrix."""
    from oracle import thc_oracle as O
    s = system
    H0, S, F = s.mean_field()
    nk = s.nk
    kw = np.full(nk, 1.0 / nk)
    Heff = H0 + F
    C, E = _eigh(Heff, S)
    mu = update_mu(0.0, nelec, E, ft.beta, kw)
    Dm = _dm(C, E, mu, ft.beta)
    Heff_mf = H_out = Heff.copy()
    Cinv = np.linalg.inv(C)
    hist = []
    for it in range(1, niter + 1):
        if hf:
            Heff = O.thc_hf(Dm, s.X, s.V, s.kpts, s.lattv, s.kp_grid, S, True, True, div,
                            madelung) + H0
        G = O.update_G(C, E, mu, ft)
        dW, _, _ = O.update_w(G, s.X, s.V, ft, s.kpts, s.lattv, s.kp_grid, s.chi_bar)
        Sigma = O.eval_Sigma_all_Rspace(G, dW, s.X, s.kpts, s.lattv, s.kp_grid)
        E_new = solve_qp_eqn(E, Sigma, Heff, C, mu, ft, qp_type, nfit, eta, tol)
        H_new = np.einsum("skai,ska,skaj->skij", np.conj(Cinv), E_new, Cinv)
        # solve_iterative: against the mean field at the first iteration, else against the
        # previous iteration's output (its checkpoint), with plain mixing
        prev = Heff_mf if it == 1 else H_out
        H_new = mixing * H_new + (1.0 - mixing) * prev
        dH = float(np.abs(H_new - prev).max())
        Heff = H_out = H_new
        E = E_new
        mu = update_mu(mu, nelec, E, ft.beta, kw)
        Dm = _dm(C, E, mu, ft.beta)
        hist.append(dict(iteration=it, E=E.copy(), mu=mu, dHeff=dH))
        if dH <= abs(conv_tol):
            break
    return dict(E=E, mu=mu, history=hist)
