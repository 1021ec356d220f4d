"""Quasiparticle-equation oracle and host logic (CPU): the Pade approximant reproduces a
rational function from its Matsubara samples, the fit-point choice, the chemical potential
and the quasiparticle rules on known functions; the library's host helpers agree with the
oracle."""
import numpy as np
import pytest

from coqui_b200 import qp as Q
from oracle import qp_oracle as QO

POLES = np.array([-0.7, -0.2, 0.45])
RES = np.array([0.05, 0.12, 0.08])


def sigma_poles(z):
    return np.sum(RES / (z - POLES))


def matsubara(n, beta=1000.0):
    return (2 * np.arange(n) + 1) * np.pi / beta


@pytest.mark.parametrize("nfit", [12, 18])
def test_pade_reproduces_a_rational_function(nfit):
    w = matsubara(200)[::11][:nfit]
    fit = QO.pade_fit(1j * w, [sigma_poles(1j * x) for x in w])
    for x in (-0.9, -0.45, 0.0, 0.3, 0.8):
        z = complex(x, 1e-3)
        assert abs(QO.pade_eval(fit, z) - sigma_poles(z)) < 1e-10 * abs(sigma_poles(z))


@pytest.mark.parametrize("niw_pos,nfit", [(24, 18), (36, 18), (30, 10), (18, 18), (50, 7)])
def test_fit_indices(niw_pos, nfit):
    idx = Q.fit_indices(niw_pos, nfit)
    assert idx == QO.fit_indices(niw_pos, nfit)
    assert len(idx) == nfit and idx[0] == 0 and idx[-1] < niw_pos
    assert all(b > a for a, b in zip(idx, idx[1:]))


def test_fit_indices_reference_example():
    # 24 positive frequencies, 18 points: 24 % 18 = 6 points with step 2, then step 1
    assert Q.fit_indices(24, 18) == [0, 2, 4, 6, 8, 10] + list(range(12, 24))


def test_update_mu_matches_oracle_and_counts_electrons():
    rng = np.random.default_rng(3)
    E = np.sort(rng.uniform(-1, 1, (1, 8, 16)), axis=2)
    kw = np.full(8, 1 / 8)
    mu = Q.update_mu(0.0, 16.0, E, 1000.0, kw)
    assert abs(mu - QO.update_mu(0.0, 16.0, E, 1000.0, kw)) < 1e-12
    assert abs(Q.compute_nelec(mu, E, 1000.0, kw) - 16.0) < 1e-8


def test_qp_rules_on_a_known_self_energy():
    # Sigma with one pole: E = V + Re Sigma(E) has a closed-form root near V
    p, r, V, mu, eta = 0.6, 0.02, -0.3, 0.0, 1e-4

    def sig(z):
        return r / (z - p)
    # roots of (E - V)(E - p) = r: the one near V
    exact = 0.5 * ((V + p) - np.sqrt((p - V) ** 2 + 4 * r))
    e_b, _ = QO.qp_eqn_bisection(V, sig, mu, V, 1e-10, eta)
    e_s, _, conv = QO.qp_eqn_secant(V, sig, mu, V, 400, 1e-12, eta)
    assert conv and abs(e_b - exact) < 1e-6 and abs(e_s - exact) < 1e-6
    e_l = QO.qp_eqn_linearized(V, sig, mu, V, eta)
    assert abs(e_l - exact) < 5e-3  # first order in the self-energy slope
