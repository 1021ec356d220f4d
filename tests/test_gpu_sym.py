"""GPU parity of the symmetry-reduced (IBZ) k-space path (coqui_b200_set_symmetry) against the
k-space oracle (oracle/sym_oracle.py), on symmetric synthetic systems: time reversal alone, and
the x <-> y mirror with a sign representation on the mirror line.

Tolerances as the full-BZ parity tests: 1e-10 max-abs (FP64 form), 1e-6 (mixed form) for Pi,
W, Sigma and 1e-6 Ha for E_c."""
import numpy as np
import pytest

from coqui_b200 import capi
from coqui_b200.iaft import IAFT as ProductIAFT
from oracle import sym_oracle as SO
from oracle import thc_oracle as O
from coqui_b200.symmetry import symmetric_system as make_sym_system

pytestmark = pytest.mark.gpu

EINVAL = -1

MODES = [(capi.FP64, 1e-10), (capi.MIXED, 1e-6)]
MODE_IDS = ["fp64", "mixed"]
CASES = [("trev", (3, 3, 1)), ("swap", (4, 4, 1))]
CASE_IDS = ["trev-331", "swap-441"]


def maxabs(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max())


class SymCase:
    def __init__(self, kind, grid, nb=8, Np=24, alat=1.0):
        self.ft = O.IAFT(1000.0, 10.0, "low")
        self.pft = ProductIAFT(1000.0, 10.0, "low")
        self.d = d = make_sym_system(kind, grid, nb, Np, self.ft, alat=alat)
        self.sym = sym = d["sym"]
        self.Pi = SO.eval_Pi_rpa_kspace(d["G_ibz"], d["X"], sym)
        self.dW = SO.update_w_kspace(d["G_ibz"], d["X"], d["V"], self.ft, sym)
        self.Sigma = SO.eval_Sigma_all_kspace(d["G_ibz"], self.dW, d["X"], sym, d["D"])
        self.e_rpa = SO.rpa_energy_kspace(d["G_ibz"], d["X"], d["V"], self.ft, sym)

    def ctx(self, mode, with_sym=True):
        d = self.d
        nk = d["sym"]["nk"]
        c = capi.Context(nk, d["X"].shape[3], d["X"].shape[2], self.ft.nt_f, self.ft.nw_b,
                         d["grid"], mode=mode)
        c.set_ir(self.pft)
        c.set_kmesh(d["kpts_lex"], d["lattv"], d["chi_lex"])
        c.set_thc(d["X_lex"], d["V_lex"])
        if with_sym:
            c.set_symmetry(self.sym, d["D"])
        return c


_cases = {}


def case(kind, grid, alat=1.0):
    key = (kind, grid, alat)
    if key not in _cases:
        _cases[key] = SymCase(kind, grid, alat=alat)
    return _cases[key]


@pytest.mark.parametrize("kind,grid", CASES, ids=CASE_IDS)
@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_ibz_pi_w_sigma_rpa(kind, grid, mode, tol):
    b = case(kind, grid)
    c = b.ctx(mode)
    G = b.d["G_ibz"]
    assert maxabs(c.eval_pi(G), b.Pi) < tol
    W, _ = c.update_w(G, want_head=False)
    assert maxabs(W, b.dW) < tol
    assert maxabs(c.eval_sigma(G), b.Sigma) < tol
    S, _ = c.gw_iteration(G)
    assert maxabs(S, b.Sigma) < tol
    # Sigma of an uploaded W
    c.set_w(b.dW)
    assert maxabs(c.eval_sigma(G), b.Sigma) < tol
    assert abs(c.rpa_energy(G) - b.e_rpa) < tol
    assert np.abs(b.Sigma).max() > 1e-3


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_ibz_sigma_with_partial_projection_cache(mode, tol):
    """The IBZ self-energy reads the projected-G cache slice by slice. With every slice, with
    the first tau chunk only (16 of 24 tau pairs on 16 k-points) and with none cached, it gives
    the same Sigma."""
    b = case("swap", (4, 4, 1))
    c = b.ctx(mode)
    G = b.d["G_ibz"]
    nk, Np, nt = b.sym["nk"], b.d["X"].shape[2], b.ft.nt_f
    nth = (nt + 1) // 2
    chunk = min(nth, max(4, -(-256 // nk)))
    assert chunk < nth  # more than one tau chunk, so one chunk is a partial cache
    slab = nk * Np * Np * (16 if mode == capi.FP64 else 8)
    res = []
    for limit in (-1, 2 * chunk * slab, 0):
        c.set_gcache_limit(limit)
        S, _ = c.gw_iteration(G)
        res.append(S)
    assert maxabs(res[0], b.Sigma) < tol
    assert maxabs(res[1], res[0]) < 1e-12
    assert maxabs(res[2], res[0]) < 1e-12


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_time_reversal_ibz_sigma_is_the_full_bz_sigma(mode, tol):
    # with time reversal the IBZ path reproduces the full-BZ path of the same context at the
    # IBZ k-points (and the RPA energy); back on the full-BZ path after set_symmetry(None)
    b = case("trev", (3, 3, 1))
    c = b.ctx(mode)
    S_ibz, _ = c.gw_iteration(b.d["G_ibz"])
    e_ibz = c.rpa_energy(b.d["G_ibz"])
    c.set_symmetry(None)
    S_full, _ = c.gw_iteration(b.d["G_lex"])
    kl = b.d["lex"][:b.sym["nk_ibz"]]
    assert maxabs(S_ibz, S_full[:, :, kl]) < 2 * tol
    assert abs(e_ibz - c.rpa_energy(b.d["G_lex"])) < 2 * tol


def test_symmetry_map_errors_are_codes():
    b = case("swap", (4, 4, 1))
    c = b.ctx(capi.FP64, with_sym=False)
    bad = dict(b.sym)
    bad["qminus"] = np.roll(b.sym["qminus"], 1)
    with pytest.raises(capi.CoquiB200Error) as e:
        c.set_symmetry(bad)
    assert e.value.code == EINVAL
    bad = dict(b.sym)
    Qs = b.sym["Qs"].copy()
    Qs[1, 0] = Qs[0, 0]  # a q-point listed twice
    bad["Qs"] = Qs
    with pytest.raises(capi.CoquiB200Error) as e:
        c.set_symmetry(bad)
    assert e.value.code == EINVAL
    bad = dict(b.sym)
    bad["kp_to_ibz"] = np.roll(b.sym["kp_to_ibz"], 1)  # the IBZ no longer first
    with pytest.raises(capi.CoquiB200Error) as e:
        c.set_symmetry(bad)
    assert e.value.code == EINVAL
    c.set_symmetry(b.sym, b.d["D"])
    with pytest.raises(capi.CoquiB200Error) as e:
        c.eval_sigma(None)  # no resident G on the IBZ route
    assert e.value.code == EINVAL
    # the context stays usable
    S, _ = c.gw_iteration(b.d["G_ibz"])
    assert maxabs(S, b.Sigma) < 1e-10


DIVS = ["gygi", "gygi_extrplt"]


@pytest.mark.parametrize("div", DIVS)
@pytest.mark.parametrize("kind,grid", CASES, ids=CASE_IDS)
@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_ibz_long_wavelength_treatments(kind, grid, mode, tol, div):
    # eps_inv_head_t over the IBZ q-points and Sigma_div_correction on the IBZ k-points;
    # a lattice constant of 8 bohr puts several |q| below the 0.8 cut of the extrapolation
    b = case(kind, grid, alat=8.0)
    d, sym = b.d, b.sym
    nqi = sym["nq_ibz"]
    rng = np.random.default_rng(3)
    chi_head = (rng.standard_normal(d["X"].shape[2]) + 1j * rng.standard_normal(d["X"].shape[2]))
    chi_head /= np.sqrt(2.0 * d["X"].shape[2])
    madelung = 0.25
    head = SO.eps_inv_head_kspace(b.dW, d["chi_bar"][:nqi], d["kpts"][:nqi], d["lattv"], b.ft,
                                  div)
    Sigma = SO.sigma_div_correction_kspace(b.Sigma, d["G_ibz"], d["X"], chi_head, head,
                                           madelung, div, nqi)
    # as in the full-BZ treatment tests: the head is compared relative to its size (it is
    # |q|^2 Omega / 4 pi chi^H W chi of the complex64 W in the mixed form), and the
    # extrapolation's sum of |weights| scales the head's and Sigma's tolerances
    Q = d["kpts"][:nqi]
    gain = 1.0
    if div == "gygi_extrplt":
        idx = O.filter_qpts(Q, 0.8, 1)
        if len(idx) >= 3:
            Qf = np.sqrt((Q[idx] ** 2).sum(axis=1))
            gain = float(sum(abs(O.extrapolate_to_q0(Qf, e)) for e in np.eye(len(idx))))
    htol = (1e-10 if mode == capi.FP64 else 1e-5) * gain * float(np.abs(head).max())
    c = b.ctx(mode)
    c.set_div_treatment(div, madelung, chi_head)
    W, h = c.update_w(d["G_ibz"], want_head=True)
    assert maxabs(W, b.dW) < tol and maxabs(h, head) < htol
    assert np.abs(head).max() > 1e-3
    assert maxabs(c.eval_sigma(d["G_ibz"]), Sigma) < tol * gain
    S, h2 = c.gw_iteration(d["G_ibz"], want_head=True)
    assert maxabs(S, Sigma) < tol * gain and maxabs(h2, h) < 1e-12
    assert maxabs(Sigma, b.Sigma) > 1e-4  # the correction is not negligible


def test_solver_mirror_takes_the_kspace_route():
    # THCData carrying the mean field's bz maps: update_w / evaluate / rpa_energy of the
    # reference-shaped interface run the IBZ route, as the reference does when
    # nqpts_ibz < nqpts (thc_gw.icc:31-32)
    from coqui_b200 import solvers
    b = case("swap", (4, 4, 1))
    d = b.d
    thc = solvers.THCData(X=d["X_lex"], V=d["V_lex"], kpts=d["kpts_lex"], lattv=d["lattv"],
                          kp_grid=d["grid"], chi_bar=d["chi_lex"], bz=b.sym,
                          bz_rotations=d["D"])
    mb = solvers.MBState(sG_tskij=d["G_ibz"])
    try:
        solvers.scr_coulomb_t(b.pft, mode=capi.FP64).update_w(mb, thc)
        assert maxabs(mb.dW_qtPQ, b.dW) < 1e-10
        gw = solvers.gw_t(b.pft, mode=capi.FP64)
        gw.evaluate(mb, thc)
        assert maxabs(mb.sSigma_tskij, b.Sigma) < 1e-10
        assert abs(gw.rpa_energy(d["G_ibz"], thc) - b.e_rpa) < 1e-10
    finally:
        solvers.clear_contexts()
