"""GPU parity of the self-consistent GW loop pieces against the FP64 oracle: Dyson equation
for G with the density matrix, Galitskii-Migdal energy, and whole loops with damping and with
commutator DIIS (scf_driver.cpp:90-173, hf = nullptr, constant mu).

The loop pieces are FP64 in both precision modes; in mixed mode the self-energy that feeds
them carries the mixed-precision error (tolerance 1e-6 as for Sigma itself).
"""
import numpy as np
import pytest

from coqui_b200 import capi
from coqui_b200.iaft import IAFT as ProductIAFT
from coqui_b200.synthetic import make_system
from oracle import thc_oracle as O

pytestmark = pytest.mark.gpu

MODES = [(capi.FP64, 1e-9), (capi.MIXED, 1e-6)]
MODE_IDS = ["fp64", "mixed"]


def maxabs(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max())


@pytest.fixture(scope="module")
def sys_():
    s = make_system(2, 8, 4, 32, seed=5)
    ft = O.IAFT(1000.0, 10.0, "low")
    H0, S, F = s.mean_field()
    return dict(s=s, ft=ft, pft=ProductIAFT(1000.0, 10.0, "low"), H0=H0, S=S, F=F, G0=s.G0(ft))


def make_ctx(d, mode):
    s, ft = d["s"], d["ft"]
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=mode)
    c.set_ir(d["pft"])
    c.set_ir_fermi(d["pft"])
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    c.set_mean_field(d["H0"], d["S"], d["F"], 0.0)
    return c


def test_dyson_g_and_gm_energy(sys_):
    d = sys_
    s, ft = d["s"], d["ft"]
    dW, _, _ = O.update_w(d["G0"], s.X, s.V, ft, s.kpts, s.lattv, s.kp_grid)
    Sigma = O.hermitize(O.eval_Sigma_all_Rspace(d["G0"], dW, s.X, s.kpts, s.lattv, s.kp_grid))
    G_ref, Dm_ref = O.dyson_G(d["H0"], d["S"], d["F"], Sigma, 0.0, ft)
    c = make_ctx(d, capi.FP64)
    G, Dm = c.dyson_g(Sigma)
    assert maxabs(G, G_ref) < 1e-10
    assert maxabs(Dm, Dm_ref) < 1e-10
    w = np.full(s.nk, 1.0 / s.nk)
    assert abs(c.gm_energy(G_ref, Sigma) - O.eval_corr_energy(G_ref, Sigma, ft, w)) < 1e-11
    c.close()


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("alg,mixing", [("damping", 0.7), ("diis", 0.2)])
def test_scgw_loop_matches_oracle(sys_, mode, tol, alg, mixing):
    d = sys_
    s, ft = d["s"], d["ft"]
    niter = 6
    hist, G_ref, S_ref = O.scgw_loop(d["G0"], s.X, s.V, d["H0"], d["S"], d["F"], 0.0, ft,
                                     s.kpts, s.lattv, s.kp_grid, niter, 0.0, alg=alg,
                                     mixing=mixing, max_subsp_size=5, diis_start=3)
    c = make_ctx(d, mode)
    c.set_iter_alg(alg, mixing, 5, 3)
    for it in range(1, niter + 1):
        st = c.scgw_iteration(it, d["G0"] if it == 1 else None)
        h = hist[it - 1]
        for key in ("e_1e", "e_hf", "e_corr"):
            assert abs(st[key] - h[key]) < tol, (it, key, st[key], h[key])
        assert abs(st["conv_Sigma"] - h["conv_Sigma"]) < tol, (it, st["conv_Sigma"], h["conv_Sigma"])
    G, S, _ = c.get_scgw_state()
    assert maxabs(G, G_ref) < tol and maxabs(S, S_ref) < tol
    c.close()


def test_diis_converges_in_fewer_iterations_than_damping(sys_):
    d = sys_
    counts = {}
    for alg, mixing in (("damping", 0.7), ("diis", 0.2)):
        c = make_ctx(d, capi.FP64)
        c.set_iter_alg(alg, mixing, 5, 3)
        for it in range(1, 30):
            st = c.scgw_iteration(it, d["G0"] if it == 1 else None)
            if st["conv_Sigma"] < 1e-8:
                break
        counts[alg] = it
        c.close()
    assert counts["diis"] < counts["damping"]
