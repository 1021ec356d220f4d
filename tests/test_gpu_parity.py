"""GPU parity: every C-ABI entry point against the FP64 oracle on seeded inputs.

Tolerances: the FP64 path agrees to 1e-10 max-abs; the mixed path (split-TF32 tensor-core
products, complex64 intermediates, FP64 Cholesky) to the stated target of 1e-6 max-abs
for Pi, W, Sigma and 1e-6 Ha for E_c.
"""
import numpy as np
import pytest

from coqui_b200 import capi, solvers
from coqui_b200.iaft import IAFT as ProductIAFT
from coqui_b200.synthetic import make_system
from oracle import thc_oracle as O

pytestmark = pytest.mark.gpu

MODES = [(capi.FP64, 1e-10), (capi.MIXED, 1e-6)]
MODE_IDS = ["fp64", "mixed"]


def maxabs(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max())


class Case:
    def __init__(self, grid, nb, nocc, Np, lam=1e4, prec="low", seed=7):
        self.s = make_system(grid, nb, nocc, Np, seed=seed)
        self.ft = O.IAFT(1000.0, lam / 1000.0, prec)
        self.pft = ProductIAFT(1000.0, lam / 1000.0, prec)
        self.G = self.s.G0(self.ft)
        s, ft = self.s, self.ft
        self.Pi = O.eval_Pi_rpa_Rspace(self.G, s.X, s.kpts, s.lattv, s.kp_grid)
        self.Pi_w = ft.tau_to_w_PHsym(self.Pi)
        self.W_w = O.dyson_W_in_place(self.Pi_w, s.V)
        self.dW, self.head, _ = O.update_w(self.G, s.X, s.V, ft, s.kpts, s.lattv, s.kp_grid,
                                           s.chi_bar)
        self.Sigma = O.eval_Sigma_all_Rspace(self.G, self.dW, s.X, s.kpts, s.lattv, s.kp_grid)
        self.e_rpa = O.rpa_energy_from_Pi_w(self.Pi_w, s.V, ft, s.nk)

    def ctx(self, mode):
        s = self.s
        c = capi.Context(s.nk, s.nb, s.Np, self.ft.nt_f, self.ft.nw_b, s.kp_grid, mode=mode)
        c.set_ir(self.pft)
        c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
        c.set_thc(s.X, s.V)
        return c


@pytest.fixture(scope="module")
def base():
    return Case(2, 16, 8, 64)


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_primary_to_aux(base, mode, tol):
    c = base.ctx(mode)
    out = c.primary_to_aux(base.G[:3])
    ref = O.primary_to_aux(base.G[:3], base.s.X[None])
    assert maxabs(out, ref) < tol


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_aux_to_primary(base, mode, tol):
    c = base.ctx(mode)
    S = base.Pi[:2, None] * 10.0  # any (nt, 1, nk, Np, Np) tensor
    out = c.aux_to_primary(S)
    ref = O.aux_to_primary(S, base.s.X[None])
    assert maxabs(out, ref) < tol * max(1.0, float(np.abs(ref).max()))


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_eval_pi(base, mode, tol):
    c = base.ctx(mode)
    assert maxabs(c.eval_pi(base.G), base.Pi) < tol


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_tau_w_transforms(base, mode, tol):
    c = base.ctx(mode)
    assert maxabs(c.tau_to_w(base.Pi), base.Pi_w) < tol
    Wt = base.ft.w_to_tau_PHsym(base.W_w)
    assert maxabs(c.w_to_tau(base.W_w), Wt) < tol


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_dyson_w(base, mode, tol):
    c = base.ctx(mode)
    assert maxabs(c.dyson_w(base.Pi_w), base.W_w) < tol


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_update_w_and_sigma(base, mode, tol):
    c = base.ctx(mode)
    W, head = c.update_w(base.G)
    assert maxabs(W, base.dW) < tol
    assert maxabs(head, base.head) < tol
    # the head is taken at the smallest nonzero |q| (find_smallest_qabs), not at q = 0
    assert np.abs(base.head).max() > 1e-3
    S = c.eval_sigma(base.G)
    assert maxabs(S, base.Sigma) < tol
    # Sigma from an uploaded W equals Sigma from the resident W
    c.set_w(base.dW)
    assert maxabs(c.eval_sigma(base.G), base.Sigma) < tol


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_gw_iteration_resident(base, mode, tol):
    c = base.ctx(mode)
    S, head = c.gw_iteration(base.G, want_head=True)
    assert maxabs(S, base.Sigma) < tol and maxabs(head, base.head) < tol
    S2, _ = c.gw_iteration(None)  # resident G
    assert maxabs(S2, S) < 1e-12
    n0 = c.kernel_launches()
    c.gw_iteration(None, want_sigma=False)
    assert c.kernel_launches() > n0


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_rpa_energy(base, mode, tol):
    c = base.ctx(mode)
    e = c.rpa_energy(base.G)
    assert abs(e - base.e_rpa) < tol
    assert abs(c.rpa_energy(None) - e) < 1e-12


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("grid,nb,nocc,Np,lam", [
    (1, 12, 6, 40, 1e4),          # Gamma only: no DFT
    ((1, 2, 3), 10, 5, 50, 1e5),  # non-cubic grid, odd nt (61), Np not a multiple of 32
    (3, 8, 4, 36, 1e4),           # 27 k-points (3-point DFT lines)
    ((2, 1, 6), 8, 4, 24, 1e4),   # 6-point lines (Good-Thomas 2 x 3) on the inner edge
    (6, 4, 2, 16, 1e4),           # 216 k-points: the compile-time cubic edge 6
    (3, 8, 4, 27, 1e4),           # register-plane kernels, 32-column tiles: 729 columns (odd, ragged last tile)
    (6, 4, 2, 18, 1e4),           # register-plane kernels, 16-column tiles: 324 columns (ragged last tile)
    ((2, 8, 2), 6, 3, 20, 1e4),   # 8-point lines (radix 2) on the middle edge
    ((1, 5, 7), 6, 3, 20, 1e4),   # 5- and 7-point lines (plain sums)
])
def test_edge_cases(mode, tol, grid, nb, nocc, Np, lam):
    cs = Case(grid, nb, nocc, Np, lam=lam, seed=11)
    c = cs.ctx(mode)
    W, head = c.update_w(cs.G)
    assert maxabs(W, cs.dW) < tol
    assert maxabs(c.eval_sigma(cs.G), cs.Sigma) < tol
    assert abs(c.rpa_energy(cs.G) - cs.e_rpa) < tol


@pytest.mark.parametrize("grid,Np", [
    (1, 300),  # groups 128 + 128 + 44: a ragged level-256 pair (256 x 44)
    ((1, 1, 2), 512),  # two doubling levels (128, 256)
])
def test_dyson_tensor_core_inverse(grid, Np):
    """Above 128 auxiliary functions the off-group blocks of C^{-1} come from the tensor
    cores (mixed mode); W must stay within the mixed tolerance of the FP64 oracle."""
    cs = Case(grid, 16, 8, Np, seed=13)
    c = cs.ctx(capi.MIXED)
    assert maxabs(c.dyson_w(cs.Pi_w), cs.W_w) < 1e-6
    W, _ = c.update_w(cs.G)
    assert maxabs(W, cs.dW) < 1e-6
    assert maxabs(c.eval_sigma(cs.G), cs.Sigma) < 1e-6
    c.close()


def test_tiled_and_one_cta_factorisations_agree(monkeypatch):
    """The tiled Cholesky (each problem over many CTAs) performs the one-CTA kernel's block
    operations in the same order: the screened interaction agrees bit for bit."""
    cs = Case(1, 16, 8, 300, seed=13)
    out = {}
    for forced in ("1", "0"):
        monkeypatch.setenv("COQUI_B200_CHOL_TILED", forced)
        c = cs.ctx(capi.MIXED)
        out[forced] = c.dyson_w(cs.Pi_w)
        c.close()
    assert np.array_equal(out["1"], out["0"])
    assert maxabs(out["1"], cs.W_w) < 1e-6


@pytest.mark.parametrize("grid,Np", [(2, 64), ((1, 1, 2), 300)])
def test_left_and_right_looking_factorisations_agree(monkeypatch, grid, Np):
    """The left-looking one-CTA factorisations (two warps; four warps with two panel row
    blocks per step, single- or double-buffered copies) start every block from I - M and
    subtract the same block products in the same order as the right-looking one (which keeps
    the running sums in global memory between block columns): W and E_c agree bit for bit."""
    cs = Case(grid, 16, 8, Np, seed=17)
    monkeypatch.setenv("COQUI_B200_CHOL_TILED", "0")
    out = {}
    forms = ("left", "right", "pair", "pair1", "pair2")
    for order in forms:
        monkeypatch.setenv("COQUI_B200_CHOL_ORDER", order)
        c = cs.ctx(capi.MIXED)
        out[order] = (c.dyson_w(cs.Pi_w), c.rpa_energy(cs.G))
        c.close()
    for order in forms[1:]:
        assert np.array_equal(out["left"][0], out[order][0]), order
        assert out["left"][1] == out[order][1], order
    assert maxabs(out["left"][0], cs.W_w) < 1e-6


def test_solver_mirror_matches_oracle(base):
    thc = solvers.THCData.from_synthetic(base.s)
    scr = solvers.scr_coulomb_t(base.pft)
    gw = solvers.gw_t(base.pft)
    mb = solvers.MBState(sG_tskij=base.G)
    scr.update_w(mb, thc)
    gw.evaluate(mb, thc)
    assert maxabs(mb.dW_qtPQ, base.dW) < 1e-6
    assert maxabs(mb.sSigma_tskij, base.Sigma) < 1e-6
    assert abs(gw.rpa_energy(base.G, thc) - base.e_rpa) < 1e-6
    solvers.clear_contexts()


def test_errors_are_codes_not_aborts(base):
    s = base.s
    c = capi.Context(s.nk, s.nb, s.Np, base.ft.nt_f, base.ft.nw_b, s.kp_grid)
    with pytest.raises(capi.CoquiB200Error) as e:
        c.update_w(base.G)  # nothing set yet
    assert e.value.code == -1
    c.set_ir(base.pft)
    with pytest.raises(capi.CoquiB200Error) as e:
        c.set_kmesh(s.kpts[::-1].copy(), s.lattv)  # not lexicographic
    assert e.value.code == -2
    bad = s.V.copy()
    bad[0] = -np.eye(s.Np)
    with pytest.raises(capi.CoquiB200Error) as e:
        c.set_thc(s.X, bad)
    assert e.value.code == -5
    # the context stays usable after errors
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    W, _ = c.update_w(base.G)
    assert maxabs(W, base.dW) < 1e-6


def test_every_tile_configuration_gives_identical_results(base):
    """Four or eight producer warps, one or two stages, 32, 64, 96 or 128 columns, one tile per
    CTA or persistent: each configuration forms the same products in the same K order, so a
    whole GW iteration agrees bit for bit whichever configuration every GEMM is pinned to."""
    c = base.ctx(capi.MIXED)
    ref = None
    try:
        for cfg in range(capi.num_tile_configs()):
            capi.set_tile_config(cfg)
            S, _ = c.gw_iteration(base.G)
            if ref is None:
                ref = S
                assert maxabs(S, base.Sigma) < 1e-6
            else:
                assert np.array_equal(S, ref), f"tile configuration {cfg}"
    finally:
        capi.set_tile_config(-1)
        c.close()


def test_autotuned_tiles_give_identical_results(base):
    """Every tile configuration forms the same products in the same K order: the tuned and
    the heuristic choice agree bit for bit."""
    capi.set_autotune(False)
    c = base.ctx(capi.MIXED)
    S0, _ = c.gw_iteration(base.G)
    capi.set_autotune(True)
    S1, _ = c.gw_iteration(base.G)
    assert capi.tuned_shapes() > 0
    assert np.array_equal(S0, S1)
    c.close()
