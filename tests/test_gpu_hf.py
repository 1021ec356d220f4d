"""GPU parity of THC Hartree-Fock (hf_t::evaluate, thc_hf.icc:17-272; HF_K_correction
hf_t.cpp:45-84) against the FP64 oracle, the reference's component check J + K = JK
(test_thc_hf.cpp:32-93), the hf_t mirror, and scGW loops that re-evaluate F each iteration
(scf_driver.cpp:94-114).

Hartree-Fock is FP64 in both precision modes (the mixed products are kept for the
imaginary-time work), so both modes meet the FP64 tolerance.
"""
import numpy as np
import pytest

from coqui_b200 import capi, solvers
from coqui_b200.iaft import IAFT as ProductIAFT
from coqui_b200.synthetic import make_system
from oracle import thc_oracle as O

pytestmark = pytest.mark.gpu

MODES = [(capi.FP64, 1e-11), (capi.MIXED, 1e-11)]
MODE_IDS = ["fp64", "mixed"]


def maxabs(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max())


def random_dm(rng, nk, nb, scale=0.25):
    A = rng.standard_normal((1, nk, nb, nb)) + 1j * rng.standard_normal((1, nk, nb, nb))
    return scale * (A + np.conj(np.swapaxes(A, -1, -2)))


def hf_ctx(s, mode):
    c = capi.Context(s.nk, s.nb, s.Np, 2, 1, s.kp_grid, mode=mode)
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    return c


CASES = [((2, 2, 2), 16, 64), ((1, 2, 3), 12, 40), (1, 24, 96), ((4, 4, 4), 32, 128)]
CASE_IDS = ["k222_nb16_np64", "k123_nb12_np40", "gamma_nb24_np96", "k444_nb32_np128"]


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("grid,nb,Np", CASES, ids=CASE_IDS)
def test_hf_matches_oracle(mode, tol, grid, nb, Np):
    s = make_system(grid, nb, nb // 2, Np, seed=11)
    rng = np.random.default_rng(4)
    Dm = random_dm(rng, s.nk, nb)
    S = np.eye(nb)[None, None] + 0.05 * random_dm(rng, s.nk, nb)
    args = (s.X, s.V, s.kpts, s.lattv, s.kp_grid, S)
    c = hf_ctx(s, mode)
    for hartree, exchange, div in ((True, True, "ignore_g0"), (True, False, "ignore_g0"),
                                   (False, True, "gygi"), (True, True, "gygi")):
        ref = O.thc_hf(Dm, *args, hartree=hartree, exchange=exchange, div=div, madelung=0.43)
        F = c.hf_evaluate(Dm, S, hartree, exchange, div, 0.43)
        scale = float(np.abs(ref).max())
        err = maxabs(F, ref) / scale
        assert err < tol, (hartree, exchange, div, err)
    c.close()


@pytest.mark.parametrize("mode", [capi.FP64, capi.MIXED], ids=MODE_IDS)
def test_hf_components_add_up(mode):
    """J + K equals the combined evaluation (test_thc_hf.cpp:61-76, 1e-8)."""
    s = make_system(2, 16, 8, 64, seed=2)
    Dm = random_dm(np.random.default_rng(1), s.nk, s.nb)
    c = hf_ctx(s, mode)
    J = c.hf_evaluate(Dm, None, True, False)
    K = c.hf_evaluate(Dm, None, False, True)
    JK = c.hf_evaluate(Dm, None, True, True)
    assert maxabs(J + K, JK) < 1e-8
    assert np.abs(c.hf_evaluate(Dm, None, False, False)).max() == 0.0
    c.close()


def test_hf_rejects_bad_arguments():
    s = make_system(1, 8, 4, 16, seed=3)
    Dm = random_dm(np.random.default_rng(0), 1, 8)
    c = hf_ctx(s, capi.FP64)
    with pytest.raises(capi.CoquiB200Error):
        c.hf_evaluate(Dm, None, True, True, "gygi", 0.3)  # gygi without the overlap
    with pytest.raises(KeyError):
        c.hf_evaluate(Dm, None, True, True, "gygi_extrplt")
    bare = capi.Context(1, 8, 16, 2, 1, (1, 1, 1), mode=capi.FP64)
    with pytest.raises(capi.CoquiB200Error):
        bare.hf_evaluate(Dm)  # no THC data yet
    bare.close()
    c.close()


def test_hf_t_mirror():
    """solvers.hf_t: the reference's constructor maps other treatments to gygi; evaluate
    overwrites sF_skij."""
    s = make_system(2, 8, 4, 32, seed=6)
    thc = solvers.THCData.from_synthetic(s)
    thc.madelung = 0.21
    rng = np.random.default_rng(7)
    Dm = random_dm(rng, s.nk, s.nb)
    S = np.eye(s.nb)[None, None] + 0.05 * random_dm(rng, s.nk, s.nb)
    hf = solvers.hf_t("gygi_extrplt", mode=capi.FP64)
    assert hf.div_treatment == "gygi"
    F = np.full((1, s.nk, s.nb, s.nb), 7.0 + 0j)
    hf.evaluate(F, Dm, thc, S)
    ref = O.thc_hf(Dm, s.X, s.V, s.kpts, s.lattv, s.kp_grid, S, div="gygi", madelung=0.21)
    assert maxabs(F, ref) < 1e-11 * np.abs(ref).max()
    solvers.clear_contexts()


@pytest.fixture(scope="module")
def loop_sys():
    s = make_system(2, 8, 4, 32, seed=5)
    ft = O.IAFT(1000.0, 10.0, "low")
    H0, S, F = s.mean_field()
    return dict(s=s, ft=ft, pft=ProductIAFT(1000.0, 10.0, "low"), H0=H0, S=S, F=F, G0=s.G0(ft))


@pytest.mark.parametrize("mode,tol", [(capi.FP64, 1e-9), (capi.MIXED, 1e-6)], ids=MODE_IDS)
@pytest.mark.parametrize("alg,mixing,div", [("damping", 0.7, "ignore_g0"),
                                            ("diis", 0.2, "gygi")])
def test_scgw_loop_with_hf_matches_oracle(loop_sys, mode, tol, alg, mixing, div):
    d = loop_sys
    s, ft = d["s"], d["ft"]
    niter = 5
    hf = dict(div=div, madelung=0.3)
    hist, G_ref, S_ref = O.scgw_loop(d["G0"], s.X, s.V, d["H0"], d["S"], d["F"], 0.0, ft,
                                     s.kpts, s.lattv, s.kp_grid, niter, 0.0, alg=alg,
                                     mixing=mixing, max_subsp_size=5, diis_start=3, hf=hf)
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=mode)
    c.set_ir(d["pft"])
    c.set_ir_fermi(d["pft"])
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    c.set_mean_field(d["H0"], d["S"], d["F"], 0.0)
    c.set_iter_alg(alg, mixing, 5, 3)
    c.set_hf(True, div, 0.3)
    for it in range(1, niter + 1):
        st = c.scgw_iteration(it, d["G0"] if it == 1 else None)
        h = hist[it - 1]
        for key in ("conv_F", "conv_Sigma", "e_1e", "e_hf", "e_corr"):
            assert abs(st[key] - h[key]) < tol, (it, key, st[key], h[key])
    G, S, _ = c.get_scgw_state()
    assert maxabs(G, G_ref) < tol and maxabs(S, S_ref) < tol
    # the loop with HF differs from the one with a fixed mean-field F
    assert abs(hist[0]["e_hf"] - O.eval_hf_energy(
        O.dm_from_G(d["G0"], ft), d["F"], d["H0"], np.full(s.nk, 1.0 / s.nk))[1]) > 1e-6
    c.close()


def test_scgw_with_hf_page_locked_start(loop_sys):
    """A page-locked starting G (copied in chunks on the copy stream) gives the same loop as
    a pageable one: the density matrix and the DIIS copy wait for every chunk."""
    import torch
    d = loop_sys
    s, ft = d["s"], d["ft"]
    G0p = torch.empty(d["G0"].shape, dtype=torch.complex128, pin_memory=True).numpy()
    G0p[...] = d["G0"]
    out = []
    for G0 in (d["G0"], G0p):
        c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=capi.FP64)
        c.set_ir(d["pft"])
        c.set_ir_fermi(d["pft"])
        c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
        c.set_thc(s.X, s.V)
        c.set_mean_field(d["H0"], d["S"], d["F"], 0.0)
        c.set_iter_alg("diis", 0.2, 5, 3)
        c.set_hf(True, "gygi", 0.3)
        out.append([c.scgw_iteration(it, G0 if it == 1 else None) for it in range(1, 4)])
        c.close()
    for a, b in zip(*out):
        for key in ("conv_F", "conv_Sigma", "e_hf", "e_corr"):
            assert abs(a[key] - b[key]) <= 1e-12 * max(1.0, abs(a[key])), (key, a[key], b[key])
