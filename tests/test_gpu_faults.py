"""Bad inputs give error codes, never aborts, and the context stays usable (host-side fault
cases; nothing here makes a GPU fault, trap or hang).

* A NaN in G: in mixed mode the projection's input check reports it (COQUI_B200_EINVAL, "G
  holds NaN or Inf values": the split-TF32 products do not carry non-finite values through
  reliably); in FP64 mode the polarizability and the dielectric matrix become NaN and the
  factorisation finds no positive pivot (COQUI_B200_ENOTHPD).
* A NaN in V or X: set_thc refuses it (COQUI_B200_EINVAL) before factorising V.
After each, the same context computes the correct result from good inputs.
"""
import numpy as np
import pytest

from coqui_b200 import capi
from coqui_b200.iaft import IAFT
from coqui_b200.synthetic import make_system
from oracle import thc_oracle as O

pytestmark = pytest.mark.gpu
ENOTHPD = -5
EINVAL = -1


@pytest.fixture(scope="module")
def case():
    s = make_system(2, 16, 8, 64, seed=41)
    ft, oft = IAFT(1000.0, 10.0, "low"), O.IAFT(1000.0, 10.0, "low")
    G = s.G0(oft)
    dW, _, _ = O.update_w(G, s.X, s.V, oft, s.kpts, s.lattv, s.kp_grid, s.chi_bar)
    Sigma = O.eval_Sigma_all_Rspace(G, dW, s.X, s.kpts, s.lattv, s.kp_grid)
    return s, ft, G, Sigma


def ctx(s, ft, mode):
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=mode)
    c.set_ir(ft)
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    return c


@pytest.mark.parametrize("mode,tol", [(capi.FP64, 1e-10), (capi.MIXED, 1e-6)], ids=["fp64", "mixed"])
def test_nan_in_g_is_an_error_code_and_the_context_recovers(case, mode, tol):
    s, ft, G, Sigma = case
    bad = G.copy()
    bad[3, 0, 1, 2, 2] = np.nan
    c = ctx(s, ft, mode)
    try:
        code = EINVAL if mode == capi.MIXED else ENOTHPD
        with pytest.raises(capi.CoquiB200Error) as e:
            c.gw_iteration(bad)
        assert e.value.code == code
        S, _ = c.gw_iteration(G)
        assert np.abs(S - Sigma).max() < tol
        # after resident-G iterations (a captured graph in mixed mode) the same holds
        c.gw_iteration(G, want_sigma=False)
        c.gw_iteration(None, want_sigma=False)
        with pytest.raises(capi.CoquiB200Error) as e:
            c.gw_iteration(bad)
        assert e.value.code == code
        with pytest.raises(capi.CoquiB200Error) as e:
            c.rpa_energy(bad)
        assert e.value.code == code
        S, _ = c.gw_iteration(G)
        assert np.abs(S - Sigma).max() < tol
    finally:
        c.close()


def test_nan_in_v_is_an_error_code(case):
    s, ft, G, Sigma = case
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=capi.MIXED)
    try:
        c.set_ir(ft)
        c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
        V = s.V.copy()
        V[1, 5, 5] = np.nan
        with pytest.raises(capi.CoquiB200Error) as e:
            c.set_thc(s.X, V)
        assert e.value.code == EINVAL
        X = s.X.copy()
        X[0, 3, 7, 2] = np.inf
        with pytest.raises(capi.CoquiB200Error) as e:
            c.set_thc(X, s.V)
        assert e.value.code == EINVAL
        c.set_thc(s.X, s.V)
        S, _ = c.gw_iteration(G)
        assert np.abs(S - Sigma).max() < 1e-6
    finally:
        c.close()
