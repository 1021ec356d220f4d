"""Oracle pinned against the reference's own fixtures (tests/golden, made by
tests/golden/make_golden.py from tests/unit_test_files/pyscf/si_kp222_krhf)."""
import os

import numpy as np
import pytest

from oracle import thc_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("prec,tol", [("high", 1e-11), ("medium", 1e-9)])
def test_iaft_transforms_match_reference_fixture(prec, tol):
    """test_iaft.cpp:46-119: tau <-> iw_n, single-w and tau -> beta^- on real GW data."""
    d = np.load(os.path.join(GOLD, f"si_kp222_gw_G_beta1000_wmax1.2_{prec}.npz"))
    ft = O.IAFT(1000.0, 1.2, prec)
    Gt, Gw, Dm = d["Gt"], d["Gw"], d["Dm"]
    assert Gt.shape[0] == ft.nt_f and Gw.shape[0] == ft.nw_f
    np.testing.assert_allclose(ft.tau_to_w(Gt, "fermi"), Gw, rtol=0, atol=tol)
    np.testing.assert_allclose(ft.w_to_tau(Gw, "fermi"), Gt, rtol=0, atol=tol)
    for n in (0, ft.nw_f // 2, ft.nw_f - 1):  # tau -> a single w
        np.testing.assert_allclose(ft.Twt_ff[n] @ Gt.reshape(ft.nt_f, -1), Gw[n].ravel(), atol=tol)
    np.testing.assert_allclose(-ft.tau_to_beta(Gt), Dm, rtol=0, atol=tol)


def test_g0_from_mos_matches_reference_fixture():
    """test_scf_common.cpp:61-96: G0(tau) from MO energies/coefficients (mu = 0.175) to 1e-8.

    The MOs are recovered from the fixture itself: G0(tau) = C g(tau) C^H with
    g_a(0+) + g_a(beta-) = -1, so B = -(G(0+) + G(beta-)) = C C^H; whitening by B = K K^H
    leaves a unitary K^-1 C that diagonalises every K^-1 G(tau) K^-H.  G0 is then rebuilt
    from (C, E) with the oracle's update_G and compared at every tau."""
    d = np.load(os.path.join(GOLD, "si_kp222_hf_G_beta1000_wmax1.2_high.npz"))
    ft = O.IAFT(1000.0, 1.2, "high")
    z = np.load(os.path.join(os.path.dirname(O.__file__), "..", "coqui_b200", "ir_data",
                             "1e4.1e-15.npz"))["T_zero_t_ff"]
    Gt = d["Gt"]  # (nt, 1, nk_kept, nb, nb)
    mu, tau = 0.175, ft.tau_mesh()
    nt, _, nk, nb, _ = Gt.shape
    C = np.zeros((1, nk, nb, nb), np.complex128)
    E = np.zeros((1, nk, nb))
    for k in range(nk):
        Gk = Gt[:, 0, k]
        B = -(np.einsum("t,tij->ij", z, Gk) + np.einsum("t,tij->ij", ft.T_beta_t_ff, Gk))
        B = 0.5 * (B + B.conj().T)
        K = np.linalg.cholesky(B)
        Ki = np.linalg.inv(K)
        Gw = np.einsum("ij,tjl,ml->tim", Ki, Gk, Ki.conj())
        _, U = np.linalg.eigh(Gw[0] + Gw[-1] + 0.37 * Gw[nt // 2])
        g = np.einsum("ia,tij,ja->ta", U.conj(), Gw, U).real  # (nt, nb)
        for a in range(nb):
            i0, i1 = np.argsort(np.abs(g[:, a]))[-2:]
            x = -np.log(g[i1, a] / g[i0, a]) / (tau[i1] - tau[i0])
            E[0, k, a] = x + mu
        C[0, k] = K @ U
    G = O.update_G(C, E, mu, ft)
    np.testing.assert_allclose(G, Gt, rtol=0, atol=1e-8)
    Dm = -ft.tau_to_beta(G)
    np.testing.assert_allclose(Dm, d["Dm"], rtol=0, atol=1e-8)
