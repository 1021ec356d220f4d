"""GPU parity of the long-wavelength treatments (div_treatment_e) against the FP64 oracle:
the eps^-1 head of update_w (eps_inv_head_t, g0_div_utils.hpp:55-111) and the self-energy's
q -> 0 correction (Sigma_div_correction, thc_gw.icc:446-526).

The k-grid is 2 x 2 x 2 on a 10-bohr cubic cell: three distinct nonzero |q| <= 0.8, so
gygi_extrplt fits its quadratic through them; gygi_extrplt_2d has two in-plane |q| and takes
the first one alone.

The head is |q|^2 Omega / 4 pi chi^H W chi (a prefactor of 8 on this cell), formed from the
complex64 W of the mixed form: it is compared relative to its size (1e-5 mixed, 1e-10 FP64).
The extrapolation to q = 0 weights its samples by up to tens (the sum of |weights|, the fit's
Lebesgue constant, is 27 here), so the extrapolated head and the Sigma it corrects carry
that factor more: tolerances scale with it.
"""
import numpy as np
import pytest

from coqui_b200 import capi, solvers
from coqui_b200.iaft import IAFT as ProductIAFT
from coqui_b200.synthetic import kgrid, make_system
from oracle import thc_oracle as O

pytestmark = pytest.mark.gpu

MODES = [(capi.FP64, 1e-10), (capi.MIXED, 1e-6)]
MODE_IDS = ["fp64", "mixed"]
DIVS = ["ignore_g0", "gygi", "gygi_extrplt", "gygi_extrplt_2d"]
MADELUNG = 0.37


def maxabs(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max())


class Case:
    def __init__(self, grid=2, L=10.0, nb=16, Np=64, seed=21):
        s = make_system(grid, nb, nb // 2, Np, seed=seed)
        s.kpts = kgrid(grid) / L
        s.lattv = np.eye(3) * L
        self.s = s
        self.ft = O.IAFT(1000.0, 10.0, "low")
        self.pft = ProductIAFT(1000.0, 10.0, "low")
        self.G = s.G0(self.ft)
        rng = np.random.default_rng(seed)
        self.chi_head = (rng.standard_normal(Np) + 1j * rng.standard_normal(Np)) / np.sqrt(Np)
        self.dW, _, self.eps_tq = O.update_w(self.G, s.X, s.V, self.ft, s.kpts, s.lattv,
                                             s.kp_grid, s.chi_bar)
        self.Sigma0 = O.eval_Sigma_all_Rspace(self.G, self.dW, s.X, s.kpts, s.lattv, s.kp_grid)

    def gain(self, div):
        """Sum of |weights| of the extrapolation to q = 0 (1 without extrapolation)."""
        if div not in ("gygi_extrplt", "gygi_extrplt_2d"):
            return 1.0
        Q = self.s.kpts
        idx = O.filter_qpts(Q, 0.8, 1, two_dim=div.endswith("2d"))
        if len(idx) < 3:
            return 1.0
        Qf = np.sqrt((Q[idx] ** 2).sum(axis=1))
        return float(sum(abs(O.extrapolate_to_q0(Qf, e)) for e in np.eye(len(idx))))

    def head(self, div):
        return O.eps_inv_head_t(self.eps_tq, self.s.kpts, self.ft, div)

    def sigma(self, div):
        return O.sigma_div_correction(self.Sigma0, self.G, self.s.X, self.chi_head,
                                      self.head(div), MADELUNG, div)

    def ctx(self, mode, div):
        s = self.s
        c = capi.Context(s.nk, s.nb, s.Np, self.ft.nt_f, self.ft.nw_b, s.kp_grid, mode=mode)
        c.set_ir(self.pft)
        c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
        c.set_thc(s.X, s.V)
        c.set_div_treatment(div, MADELUNG, self.chi_head)
        return c


@pytest.fixture(scope="module")
def case():
    return Case()


def test_oracle_case_exercises_every_branch(case):
    Q = case.s.kpts
    assert len(O.filter_qpts(Q, 0.8, 1)) == 3
    assert len(O.filter_qpts(Q, 0.8, 1, two_dim=True)) == 2
    heads = {d: case.head(d) for d in DIVS}
    assert maxabs(heads["gygi_extrplt"], heads["gygi"]) > 1e-6  # the fit moves the head
    assert 20 < case.gain("gygi_extrplt") < 40 and case.gain("gygi_extrplt_2d") == 1.0
    assert maxabs(case.sigma("gygi"), case.Sigma0) > 1e-6


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("div", DIVS)
def test_head_and_sigma_match_oracle(case, mode, tol, div):
    c = case.ctx(mode, div)
    W, head = c.update_w(case.G)
    ref = case.head(div)
    hrel = 1e-10 if mode == capi.FP64 else 1e-5
    assert maxabs(head, ref) < hrel * case.gain(div) * float(np.abs(ref).max())
    tol = tol * case.gain(div)
    S = c.eval_sigma(case.G)
    assert maxabs(S, case.sigma(div)) < tol
    # the same through one call with a head out, and with W uploaded instead of computed
    S2, head2 = c.gw_iteration(case.G, want_head=True)
    assert maxabs(S2, S) < 1e-12 and maxabs(head2, head) < 1e-12
    c.set_w(case.dW)
    assert maxabs(c.eval_sigma(case.G), case.sigma(div)) < tol
    c.close()


def test_treatment_change_on_the_same_w(case):
    """Changing the treatment between self-energies of one W re-selects the head (W is
    brought back to q-space once when an earlier call left it in R)."""
    c = case.ctx(capi.FP64, "ignore_g0")
    c.update_w(case.G, want_w=False, want_head=False)
    assert maxabs(c.eval_sigma(case.G), case.sigma("ignore_g0")) < 1e-10
    c.set_div_treatment("gygi_extrplt", MADELUNG)  # chi_head kept
    assert maxabs(c.eval_sigma(case.G), case.sigma("gygi_extrplt")) < 1e-10
    c.close()


def test_page_locked_buffers_with_correction(case):
    """With a treatment set the iteration takes the plain path (the head is needed on the
    host between W and Sigma): page-locked buffers give the same Sigma."""
    import torch
    c = case.ctx(capi.MIXED, "gygi")
    Gp = torch.empty(case.G.shape, dtype=torch.complex128, pin_memory=True).numpy()
    Gp[...] = case.G
    Sp = torch.empty(case.G.shape, dtype=torch.complex128, pin_memory=True).numpy()
    ref = case.sigma("gygi")
    for _ in range(3):
        c.gw_iteration(Gp, sigma_out=Sp)
        assert maxabs(Sp, ref) < 1e-6
    c.close()


def test_one_q_point_is_ignore_g0():
    """With one q-point every treatment acts as ignore_g0 (thc_gw.icc:454-458)."""
    s = make_system(1, 12, 6, 48, seed=8)
    ft = O.IAFT(1000.0, 10.0, "low")
    G = s.G0(ft)
    out = []
    for div in ("ignore_g0", "gygi_extrplt"):
        c = capi.Context(1, s.nb, s.Np, ft.nt_f, ft.nw_b, (1, 1, 1), mode=capi.FP64)
        c.set_ir(ProductIAFT(1000.0, 10.0, "low"))
        c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
        c.set_thc(s.X, s.V)
        c.set_div_treatment(div, 0.5, np.ones(s.Np))
        out.append(c.gw_iteration(G, want_head=True))
        c.close()
    assert maxabs(out[0][0], out[1][0]) == 0.0 and maxabs(out[0][1], out[1][1]) == 0.0


def test_treatment_errors(case):
    s = case.s
    c = capi.Context(s.nk, s.nb, s.Np, case.ft.nt_f, case.ft.nw_b, s.kp_grid, mode=capi.FP64)
    c.set_ir(case.pft)
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    with pytest.raises(KeyError):
        c.set_div_treatment("ewald")
    assert c.lib.coqui_b200_set_div_treatment(c.h, 7, 0.0, None) == -1
    c.set_div_treatment("gygi", 0.3)  # no chi_head yet
    c.update_w(case.G, want_w=False, want_head=False)
    with pytest.raises(capi.CoquiB200Error):
        c.eval_sigma(case.G)
    c.close()
    # no q-point within 0.8 for the extrapolation: lattice constant 1 bohr
    s1 = make_system(2, 8, 4, 32, seed=3)
    c = capi.Context(s1.nk, s1.nb, s1.Np, case.ft.nt_f, case.ft.nw_b, s1.kp_grid, mode=capi.FP64)
    c.set_ir(case.pft)
    c.set_kmesh(s1.kpts, s1.lattv, s1.chi_bar)
    c.set_thc(s1.X, s1.V)
    c.set_div_treatment("gygi_extrplt", 0.3, np.ones(s1.Np))
    with pytest.raises(capi.CoquiB200Error):
        c.update_w(s1.G0(case.ft), want_w=False)
    c.close()


def test_solver_mirror_with_treatment(case):
    s = case.s
    thc = solvers.THCData(X=s.X, V=s.V, kpts=s.kpts, lattv=s.lattv, kp_grid=s.kp_grid,
                          chi_bar=s.chi_bar, madelung=MADELUNG, chi_head=case.chi_head)
    mb = solvers.MBState(sG_tskij=case.G)
    solvers.scr_coulomb_t(case.pft, div_treatment="gygi_extrplt", mode=capi.FP64).update_w(mb, thc)
    assert maxabs(mb.eps_inv_head, case.head("gygi_extrplt")) < 1e-10
    solvers.gw_t(case.pft, div_treatment="gygi_extrplt", mode=capi.FP64).evaluate(mb, thc)
    assert maxabs(mb.sSigma_tskij, case.sigma("gygi_extrplt")) < 1e-10
    solvers.clear_contexts()
