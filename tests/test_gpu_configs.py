"""GPU parity at the benchmark's own configurations, against the FP64 oracle.

* 2x2x2 k, 16 orbitals (8 occupied), N_mu = 128, beta = 1000, Lambda = 1e4 ("low", 48 tau):
  the RPA configuration the oracle runs in seconds.  Every stage of the path is compared:
  Pi(tau), Pi(iW), W(iW), dW_qtPQ and the dielectric head, Sigma and E_c.
* 4x4x4 k, 64 orbitals (24 occupied), N_mu = 512 (the G0W0 configuration): dW_qtPQ, Sigma
  and E_c of the whole iteration.  The oracle takes about a minute of host time.

Tolerances: FP64 mode 1e-10 max-abs (E_c 1e-10 Ha); mixed mode (split-TF32 products,
complex64 intermediates, FP64 factorisations) 1e-6 max-abs for Pi, W and Sigma and 1e-6 Ha
for E_c -- the targets the path is built to.
"""
import numpy as np
import pytest

from coqui_b200 import capi
from coqui_b200.iaft import IAFT as ProductIAFT
from coqui_b200.synthetic import WORKLOADS, make_system
from oracle import thc_oracle as O

pytestmark = pytest.mark.gpu

TOL = {capi.FP64: 1e-10, capi.MIXED: 1e-6}
MODES = [capi.FP64, capi.MIXED]
IDS = ["fp64", "mixed"]


def maxabs(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max())


class Reference:
    """The oracle's whole RPA/GW step on one named workload (intermediates kept only where a
    test compares them)."""

    def __init__(self, name, keep_stages):
        w = WORKLOADS[name]
        self.s = make_system(w["n"], w["nb"], w["nocc"], w["Np"], beta=w["beta"], seed=2024)
        self.ft = O.IAFT(w["beta"], w["lam"] / w["beta"], w["prec"])
        self.pft = ProductIAFT(w["beta"], w["lam"] / w["beta"], w["prec"])
        s, ft = self.s, self.ft
        self.G = s.G0(ft)
        Pi = O.eval_Pi_rpa_Rspace(self.G, s.X, s.kpts, s.lattv, s.kp_grid)
        Pi_w = ft.tau_to_w_PHsym(Pi)
        self.e_rpa = O.rpa_energy_from_Pi_w(Pi_w, s.V, ft, s.nk)
        W_w = O.dyson_W_in_place(Pi_w, s.V)
        if keep_stages:
            self.Pi, self.Pi_w, self.W_w = Pi, Pi_w, W_w
        del Pi, Pi_w
        W_t = ft.w_to_tau_PHsym(W_w)
        del W_w
        eps = O.eval_eps_inv_q(W_t, s.chi_bar, s.kpts, s.lattv)
        self.head = O.eps_inv_head_t(eps, s.kpts, ft, "ignore_g0")
        self.dW = np.ascontiguousarray(np.swapaxes(W_t, 0, 1))  # scr_coulomb_t.cpp:73-86
        del W_t
        self.Sigma = O.eval_Sigma_all_Rspace(self.G, self.dW, s.X, s.kpts, s.lattv, s.kp_grid)

    def ctx(self, mode):
        s = self.s
        c = capi.Context(s.nk, s.nb, s.Np, self.ft.nt_f, self.ft.nw_b, s.kp_grid, mode=mode)
        c.set_ir(self.pft)
        c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
        c.set_thc(s.X, s.V)
        return c


@pytest.fixture(scope="module")
def rpa_k2():
    return Reference("rpa_k2_nb16_np128", keep_stages=True)


@pytest.fixture(scope="module")
def g0w0_k4():
    return Reference("g0w0_k4_nb64_np512", keep_stages=False)


@pytest.mark.parametrize("mode", MODES, ids=IDS)
def test_rpa_k2_nb16_np128_every_stage(rpa_k2, mode):
    r, tol = rpa_k2, TOL[mode]
    c = r.ctx(mode)
    try:
        assert maxabs(c.eval_pi(r.G), r.Pi) < tol
        assert maxabs(c.tau_to_w(r.Pi), r.Pi_w) < tol
        assert maxabs(c.dyson_w(r.Pi_w), r.W_w) < tol
        W, head = c.update_w(r.G)
        assert maxabs(W, r.dW) < tol
        assert maxabs(head, r.head) < tol
        assert np.abs(r.head).max() > 1e-3  # the head is taken at the smallest nonzero |q|
        assert maxabs(c.eval_sigma(r.G), r.Sigma) < tol
        S, _ = c.gw_iteration(r.G)
        assert maxabs(S, r.Sigma) < tol
        assert abs(c.rpa_energy(r.G) - r.e_rpa) < tol
    finally:
        c.close()


@pytest.mark.parametrize("mode", MODES, ids=IDS)
def test_g0w0_k4_nb64_np512_whole_iteration(g0w0_k4, mode):
    r, tol = g0w0_k4, TOL[mode]
    c = r.ctx(mode)
    try:
        W, head = c.update_w(r.G)
        assert maxabs(W, r.dW) < tol
        assert maxabs(head, r.head) < tol
        del W
        S = c.eval_sigma(r.G)
        assert maxabs(S, r.Sigma) < tol
        assert abs(c.rpa_energy(r.G) - r.e_rpa) < tol
    finally:
        c.close()
