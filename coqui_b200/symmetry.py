"""Brillouin-zone symmetry maps for the IBZ k-space path, and symmetric synthetic inputs.

``bz_symmetry`` builds the lists that CoQui's mean field carries in ``bz_symm``
(src/mean_field/symmetry/bz_symmetry.hpp:48-333 with ``generate_qsymm_maps``,
src/utilities/symmetry.hpp:498-590) for a Gamma-centred grid and operations given as integer
matrices on the grid's crystal coordinates: the 1st-BZ k list with the IBZ points first (each
the lexicographically first point of its orbit), the time-reversal images of the IBZ appended,
then the images of the operation that adds the most new points, time-reversal points moved to
the end; ``kp_trev_pair``; the q maps of a Gamma-centred grid (Qpts = kpts, qp_to_ibz =
kp_to_ibz); ``qsymms``, ``nq_per_s``, ``Qs``, ``ks_to_k``; and ``qk_to_k2`` / ``qminus``
(kpoint_utils.hpp:27-90).  ``ops[s]`` generates the images (the reference's R^-1 transposed);
index 0 is the identity.  The result feeds :meth:`coqui_b200.capi.Context.set_symmetry` (its
``lex`` entry is each k-point's position in the lexicographic grid).

``symmetric_system`` draws seeded THC inputs with a symmetry (time reversal, or the x <-> y
mirror of an n x n x m grid with a sign representation on the mirror line) in both the
reference's k order (for the IBZ path) and the lexicographic order (for the full-BZ path).
"""
from __future__ import annotations

import numpy as np

SWAP = np.array([[0, 1, 0], [1, 0, 0], [0, 0, 1]])


def _key(m, grid):
    return tuple(int(v) % int(g) for v, g in zip(m, grid))


def bz_symmetry(kp_grid, ops, use_trev):
    """bz_symm lists of a Gamma-centred grid (see the module docstring).  Returns a dict with
    integer crystal coordinates ``kc`` (nk, 3) in the reference's order, ``lex``, ``nk``,
    ``nk_ibz``, ``nq_ibz`` and the maps ``kp_to_ibz``, ``kp_symm``, ``kp_trev``,
    ``kp_trev_pair``, ``qp_to_ibz``, ``qp_symm``, ``qp_trev``, ``qsymms``, ``nq_per_s``,
    ``Qs``, ``ks_to_k``, ``qk_to_k2``, ``qminus``."""
    grid = tuple(int(g) for g in kp_grid)
    ops = [np.asarray(M, np.int64) for M in ops]
    nsymm = len(ops)
    allk = [(a, b, c) for a in range(grid[0]) for b in range(grid[1]) for c in range(grid[2])]

    def act(M, k):
        return _key(M @ np.asarray(k), grid)

    def neg(k):
        return _key(-np.asarray(k), grid)

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
    kplist, kp_s, kp_ibz, trev = list(ibz), [0] * nk_ibz, list(range(nk_ibz)), [False] * nk_ibz
    known = set(kplist)
    k_gamma = ibz.index((0, 0, 0))
    if nsymm > 1 or use_trev:
        if use_trev:
            for j in range(nk_ibz):
                kp = neg(kplist[j])
                if j != k_gamma and kp not in known:
                    kplist.append(kp)
                    known.add(kp)
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
                v, vs, idx, tf = [], set(), [], []
                for j in range(nk_ibz):
                    if j == k_gamma:
                        continue
                    for t in ((False, True) if use_trev else (False,)):
                        kp = act(ops[s], kplist[j])
                        kp = neg(kp) if t else kp
                        if kp not in known and kp not in vs:
                            v.append(kp)
                            vs.add(kp)
                            idx.append(j)
                            tf.append(t)
                if v and (best is None or len(v) > len(best[1])):
                    best = (s, v, idx, tf)
            if best is None:
                break
            s, v, idx, tf = best
            done[s] = True
            kplist += v
            known |= set(v)
            kp_s += [s] * len(v)
            kp_ibz += idx
            trev += tf
    nk = len(kplist)
    if nk != len(allk):
        raise ValueError("the operations do not generate the whole grid")
    order = [i for i in range(nk) if not trev[i]] + [i for i in range(nk) if trev[i]]
    kplist = [kplist[i] for i in order]
    kp_s = np.array([kp_s[i] for i in order], np.int64)
    kp_ibz = np.array([kp_ibz[i] for i in order], np.int64)
    trev = np.array([trev[i] for i in order], bool)
    index = {k: i for i, k in enumerate(kplist)}
    ntrev = int(trev.sum())
    pair = np.full(nk, -1, np.int64)
    for ik in range(nk - ntrev, nk):
        n = index[neg(kplist[ik])]
        if trev[n] or kp_s[n] != kp_s[ik] or kp_ibz[n] != kp_ibz[ik]:
            raise ValueError("time-reversal partner not found")
        pair[ik], pair[n] = n, ik
    if nsymm == 1 and not use_trev:
        qp_symm, qp_trev, qp_to_ibz, nq_ibz = (np.zeros(nk, np.int64), np.zeros(nk, bool),
                                              np.arange(nk), nk)
    else:
        qp_symm, qp_trev, qp_to_ibz, nq_ibz = kp_s.copy(), trev.copy(), kp_ibz.copy(), nk_ibz
    unique = []
    for s in qp_symm:
        if int(s) not in unique:
            unique.append(int(s))
    if len(unique) == 1 and unique[0] == 0 and not use_trev:
        qsymms, nq_per_s = np.array([0]), np.array([nk])
        ks_to_k = np.arange(nk)[None, :].copy()
        Qs = np.zeros((1, 2 * nq_ibz), np.int64)
        Qs[0, :nq_ibz] = np.arange(nq_ibz)
    else:
        qsymms = np.array(unique, np.int64)
        nq_per_s = np.array([int((qp_symm == s).sum()) for s in unique], np.int64)
        ks_to_k = np.zeros((len(unique), nk), np.int64)
        Qs = np.zeros((len(unique), 2 * nq_ibz), np.int64)
        for i, s in enumerate(unique):
            js = np.flatnonzero(qp_symm == s)
            Qs[i, :len(js)] = js
            Rt = np.rint(np.linalg.inv(ops[s])).astype(np.int64)
            for ik in range(nk):
                ks_to_k[i, ik] = index[act(Rt, kplist[ik])]
    kc = np.array(kplist, np.int64)
    g = np.array(grid)
    lex_of = lambda m: int(((m[..., 0] % g[0]) * g[1] + m[..., 1] % g[1]) * g[2] + m[..., 2] % g[2])  # noqa: E731
    inv = np.empty(nk, np.int64)
    lex = np.array([lex_of(k) for k in kc], np.int64)
    inv[lex] = np.arange(nk)
    qk_to_k2 = np.array([[inv[lex_of(kc[k] - kc[q])] for k in range(nk)] for q in range(nk)],
                        np.int64)
    qminus = np.array([inv[lex_of(-kc[q])] for q in range(nk)], np.int64)
    return dict(kc=kc, lex=lex, nk=nk, nk_ibz=nk_ibz, nq_ibz=nq_ibz, kp_to_ibz=kp_ibz,
                kp_symm=kp_s, kp_trev=trev, kp_trev_pair=pair, qp_to_ibz=qp_to_ibz,
                qp_symm=qp_symm, qp_trev=qp_trev, qsymms=qsymms, nq_per_s=nq_per_s, Qs=Qs,
                ks_to_k=ks_to_k, qk_to_k2=qk_to_k2, qminus=qminus, grid=grid)


def _cn(rng, shape, scale=1.0):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * (scale / np.sqrt(2.0))


def _hpd(rng, Np):
    Z = _cn(rng, (Np, Np), 1.0 / np.sqrt(Np))
    return Z @ Z.conj().T + 0.05 * np.eye(Np)


def green_tau(H0_kij, ft, mu=0.0):
    """G_tkij(tau) of the one-body Hamiltonians H0 (orthonormal basis) at chemical potential mu,
    g(e, tau) written without overflow on either side of mu (qp_scf_common.cpp:82-118)."""
    E, C = np.linalg.eigh(H0_kij)
    tau = ft.tau_mesh()[:, None, None]
    x = (E - mu)[None]
    pos = x > 0
    xp, xn = np.where(pos, x, 0.0), np.where(pos, 0.0, x)
    g = np.where(pos, -np.exp(-xp * tau) / (1.0 + np.exp(-xp * ft.beta)),
                 -np.exp(xn * (ft.beta - tau)) / (1.0 + np.exp(xn * ft.beta)))
    return np.einsum("kia,tka,kja->tkij", C, g, np.conj(C))


def symmetric_system(kind, kp_grid, nb, Np, ft, seed=7, mu=0.0, alat=1.0):
    """Seeded THC inputs with a symmetry on a cubic lattice (lattv = alat I):

    * ``"trev"``: time reversal alone: X^{-k} = conj(X^k), H0^{-k} = conj(H0^k); at k = -k
      X and H0 are real;
    * ``"swap"``: the mirror x <-> y of an n x n x m grid, used without time reversal.  The
      auxiliary points come in mirror pairs (P, pi(P)) plus two points on the plane;
      X^{Sk}_P = X^k_{pi(P)} and H0^{Sk} = H0^k; on the mirror line X^k_{pi(P)} = X^k_P D_k
      with D_k = diag(+-1) (points on the plane carry only the even orbitals) and H0^k
      commutes with D_k, which is then the rotation d[S, k].

    V is a physical Coulomb matrix in both, V^{-q} = conj(V^q), with the model's symmetry:
    one random Hermitian positive definite matrix per orbit of {E, S} x {1, T}, averaged over
    the stabilizer of the orbit's first point.  The chi-bar heads are CN(0, 1/Np) per q-point.
    Returns the maps (``sym``), D, X / V / G_ibz / chi_bar / kpts in the reference's order, and
    X_lex / V_lex / G_lex (G unfolded to every k-point with the reference's rule) / chi_lex /
    kpts_lex in lexicographic order."""
    rng = np.random.default_rng(seed)
    grid = tuple(int(g) for g in kp_grid)
    if kind == "trev":
        sym = bz_symmetry(grid, [np.eye(3, dtype=int)], True)
    elif kind == "swap":
        if grid[0] != grid[1]:
            raise ValueError("the mirror needs an n x n x m grid")
        sym = bz_symmetry(grid, [np.eye(3, dtype=int), SWAP], False)
    else:
        raise ValueError(kind)
    nk, nk_ibz, kc = sym["nk"], sym["nk_ibz"], sym["kc"]
    nfix = 2 if kind == "swap" else 0
    npair = (Np - nfix) // 2
    pi = np.arange(Np)
    if kind == "swap":
        pi[0:2 * npair:2], pi[1:2 * npair:2] = np.arange(1, 2 * npair, 2), np.arange(0, 2 * npair, 2)
    X = np.zeros((nk, Np, nb), np.complex128)
    H0 = np.zeros((nk, nb, nb), np.complex128)
    V = np.zeros((nk, Np, Np), np.complex128)
    nsym = len(sym["qsymms"])
    D = np.broadcast_to(np.eye(nb, dtype=np.complex128), (nsym, nk_ibz, nb, nb)).copy()
    eps = np.sort(rng.uniform(-1.0, 1.0, nb))
    for j in range(nk_ibz):
        k = kc[j]
        Xj = _cn(rng, (Np, nb), 1.0 / np.sqrt(Np))
        A = _cn(rng, (nb, nb), 0.2)
        Hj = 0.5 * (A + A.conj().T) + np.diag(eps)
        if kind == "trev" and np.all((-k) % np.array(grid) == k):
            Xj, Hj = Xj.real.astype(np.complex128), Hj.real.astype(np.complex128)
        if kind == "swap" and k[0] == k[1]:
            s = np.where(rng.random(nb) < 0.5, -1.0, 1.0)
            s[0], s[-1] = 1.0, -1.0
            Dj = np.diag(s).astype(np.complex128)
            Xj[1:2 * npair:2] = Xj[0:2 * npair:2] @ Dj
            Xj[2 * npair:] *= (s > 0)
            Hj = 0.5 * (Hj + Dj @ Hj @ Dj)
            D[1, j] = Dj
        X[j], H0[j] = Xj, Hj
    for i in range(nk_ibz, nk):
        j = sym["kp_to_ibz"][i]
        if kind == "trev":
            X[i], H0[i] = np.conj(X[j]), np.conj(H0[j])
        else:
            X[i], H0[i] = X[j][pi], H0[j]
    mirror = [(np.eye(3, dtype=int), np.arange(Np))] + ([(SWAP, pi)] if kind == "swap" else [])
    group = [(M, p, t) for (M, p) in mirror for t in (False, True)]
    kidx = {tuple(int(v) for v in kc[i]): i for i in range(nk)}
    done = np.zeros(nk, bool)

    def act(A, p, t):
        B = A[np.ix_(p, p)]
        return np.conj(B) if t else B

    for i in range(nk):
        if done[i]:
            continue
        imgs = [(kidx[tuple(int(v) for v in ((M @ kc[i]) * (-1 if t else 1)) % np.array(grid))], p, t)
                for M, p, t in group]
        V0 = _hpd(rng, Np)
        stab = [(p, t) for (n, p, t) in imgs if n == i]
        Vi = sum(act(V0, p, t) for p, t in stab) / len(stab)
        for n, p, t in imgs:
            V[n] = act(Vi, p, t)
            done[n] = True
    chi = _cn(rng, (nk, Np), 1.0 / np.sqrt(Np))
    G_ibz = green_tau(H0[:nk_ibz], ft, mu)[:, None]  # (nt, 1, nk_ibz, nb, nb)
    lex = sym["lex"]
    G_full = G_ibz[:, :, sym["kp_to_ibz"]]
    tr = np.asarray(sym["kp_trev"], bool)
    G_full = np.where(tr[None, None, :, None, None], np.swapaxes(G_full, -1, -2), G_full)
    inv = np.empty(nk, np.int64)
    inv[lex] = np.arange(nk)
    kpts = 2.0 * np.pi * kc / (np.array(grid, np.float64) * alat)
    return dict(sym=sym, D=D, X=X[None], V=V, G_ibz=G_ibz, lattv=alat * np.eye(3), grid=grid,
                chi_bar=chi, kpts=kpts, X_lex=X[inv][None], V_lex=V[inv],
                G_lex=np.ascontiguousarray(G_full[:, :, inv]), chi_lex=chi[inv],
                kpts_lex=kpts[inv], lex=lex, inv=inv, pi=pi)
