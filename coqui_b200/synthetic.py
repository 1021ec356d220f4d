"""Seeded synthetic THC mean-field systems.

The reference builds its THC collocation X and Coulomb matrix V by ISDF from a
mean-field calculation (``src/methods/ERI/thc.h``).  The workloads here instead draw
them from fixed distributions, with the reference's array layouts
(``src/methods/ERI/thc_reader_t.hpp:532-541``: X is (ns*npol, nk, Np, nb);
``:714-751``: V is (nq, Np, Np)):

* cubic lattice ``lattv = I`` (bohr), Gamma-centred ``n x n x n`` k-grid in lexicographic
  order, ``kpts = 2 pi (i, j, l) / n``; no symmetry, nq = nk, Qpts = kpts;
* ``X^k_{mu i} ~ CN(0, 1) / sqrt(Np)``;
* ``V^q = Z^q Z^q^H + 1e-3 I`` with ``Z^q ~ CN(0, 1/Np)``, Hermitian positive definite;
* orbital energies uniform on [-1, -0.1] (occupied) and [0.1, 1] (virtual), MO
  coefficients C = I, mu = 0; G0(tau) from them as in ``qp_scf_common.cpp:82-118``;
* chi-bar heads ``chi_bar_qP ~ CN(0,1)/sqrt(Np)`` (the reference's
  ``thc_reader_t::basis_bar_head``), used only by the dielectric-head diagnostic.

CN(0, s^2) means (a + i b) * s / sqrt(2) with a, b ~ N(0, 1).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .iaft import IAFT


def _cn(rng, shape, scale=1.0):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * (scale / np.sqrt(2.0))


@dataclass
class SyntheticSystem:
    kp_grid: tuple
    nb: int
    nocc: int
    Np: int
    beta: float
    kpts: np.ndarray
    lattv: np.ndarray
    X: np.ndarray  # (1, nk, Np, nb) complex128
    V: np.ndarray  # (nq, Np, Np) complex128
    eps: np.ndarray  # (1, nk, nb) float64
    chi_bar: np.ndarray  # (nq, Np) complex128
    mu: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def nk(self) -> int:
        return int(self.kpts.shape[0])

    def mean_field(self):
        """(H0, S, F) of the synthetic mean field, each (1, nk, nb, nb) complex128: H0 holds
        the orbital energies (C = I), S = I, and the Fock part is zero (the loop runs with a
        fixed mean-field Fock, scf_driver.cpp:94 with hf = nullptr)."""
        nk, nb = self.eps.shape[1], self.nb
        H0 = np.zeros((1, nk, nb, nb), np.complex128)
        idx = np.arange(nb)
        H0[0][:, idx, idx] = self.eps[0]
        S = np.broadcast_to(np.eye(nb, dtype=np.complex128), (1, nk, nb, nb)).copy()
        return H0, S, np.zeros_like(H0)

    def G0(self, ft: IAFT) -> np.ndarray:
        """G0_tskij(tau) for C = I (diagonal), qp_scf_common.cpp:86-93."""
        tau = ft.tau_mesh()
        x = self.eps[0] - self.mu  # (nk, nb)
        t = tau[:, None, None]
        pos = x > 0
        xp = np.where(pos, x, 0.0)[None]
        xn = np.where(pos, 0.0, x)[None]
        g_pos = -np.exp(-xp * t) / (1.0 + np.exp(-xp * self.beta))
        g_neg = -np.exp(xn * (self.beta - t)) / (1.0 + np.exp(xn * self.beta))
        g = np.where(pos[None], g_pos, g_neg)  # (nt, nk, nb)
        nt, nk, nb = g.shape
        G = np.zeros((nt, 1, nk, nb, nb), np.complex128)
        ii = np.arange(nb)
        G[:, 0, :, ii, ii] = np.moveaxis(g, 2, 0)
        return G


def kgrid(n):
    """Gamma-centred grid in lexicographic order, cartesian 2 pi (i/n0, j/n1, l/n2) (lattv = I).

    ``n`` is an int (n x n x n) or a 3-tuple."""
    n0, n1, n2 = (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)
    idx = np.array([(i / n0, j / n1, l / n2) for i in range(n0) for j in range(n1)
                    for l in range(n2)], np.float64)
    return 2.0 * np.pi * idx


def make_system(n, nb: int, nocc: int, Np: int, beta: float = 1000.0, seed: int = 0,
                gamma_only: bool = False) -> SyntheticSystem:
    """Seeded system on an n x n x n (int n) or n0 x n1 x n2 (tuple n) k-grid."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if gamma_only:
        n = 1
    grid = (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)
    kpts = kgrid(grid)
    nk = kpts.shape[0]
    X = _cn(rng, (1, nk, Np, nb), 1.0 / np.sqrt(Np))
    Z = _cn(rng, (nk, Np, Np), 1.0 / np.sqrt(Np))
    V = Z @ np.conj(np.swapaxes(Z, -1, -2)) + 1e-3 * np.eye(Np)[None]
    occ = rng.uniform(-1.0, -0.1, size=(1, nk, nocc))
    vir = rng.uniform(0.1, 1.0, size=(1, nk, nb - nocc))
    eps = np.concatenate([occ, vir], axis=2)
    chi_bar = _cn(rng, (nk, Np), 1.0 / np.sqrt(Np))
    return SyntheticSystem(kp_grid=grid, nb=nb, nocc=nocc, Np=Np, beta=beta,
                           kpts=kpts, lattv=np.eye(3), X=X, V=V, eps=eps, chi_bar=chi_bar,
                           meta=dict(seed=seed))


# Named workloads (k-grid edge, nb, nocc, Np, beta, Lambda, prec).
WORKLOADS = {
    "rpa_k2_nb16_np128": dict(n=2, nb=16, nocc=8, Np=128, beta=1000.0, lam=1e4, prec="low"),
    "g0w0_k4_nb64_np512": dict(n=4, nb=64, nocc=24, Np=512, beta=1000.0, lam=1e4, prec="low"),
    # same orbitals / N_mu on a 2x2x2 grid: the small case used for kernel profiles
    "g0w0_k2_nb64_np512": dict(n=2, nb=64, nocc=24, Np=512, beta=1000.0, lam=1e4, prec="low"),
    # 64 k-points at a smaller N_mu: the case used for profiles of the k <-> R kernels
    "g0w0_k4_nb48_np384": dict(n=4, nb=48, nocc=24, Np=384, beta=1000.0, lam=1e4, prec="low"),
    # 6x6x6 k-points (the headline grid's column kernels) at a small N_mu and IR grid: a
    # 143 MB tau slice (larger than L2) in about 10 GB of device memory, for kernel profiles
    "g0w0_k6_nb32_np288": dict(n=6, nb=32, nocc=16, Np=288, beta=100.0, lam=1e3, prec="low"),
    "rpa_gw_k6_nb96_np1024": dict(n=6, nb=96, nocc=48, Np=1024, beta=1000.0, lam=1e5, prec="low"),
    "scgw_k3_nb48_np384": dict(n=3, nb=48, nocc=24, Np=384, beta=1000.0, lam=1e4, prec="low"),
}
