"""Shipped IR tables: sizes and identities pinned by the reference's own tests
(src/numerics/imag_axes_ft/ir/tests/test_ir.cpp:16-39,
 src/numerics/imag_axes_ft/tests/test_iaft.cpp:17-44)."""
import numpy as np
import pytest

from coqui_b200.iaft import IAFT as ProductIAFT
from oracle.thc_oracle import IAFT


def test_lambda_1e5_high_sizes_and_identity():
    ft = IAFT(1000.0, 12.0, "high")  # beta*wmax = 12000 -> Lambda = 1e5
    assert ft.lam == 1e5
    assert (ft.nt_f, ft.nw_f, ft.nt_b, ft.nw_b) == (137, 138, 137, 137)
    assert ft.Ttw_ff.shape == (137, 138) and ft.Twt_ff.shape == (138, 137)
    assert ft.Ttw_bb.shape == (137, 137) and ft.Twt_bb.shape == (137, 137)
    np.testing.assert_allclose(ft.Ttw_ff @ ft.Twt_ff, np.eye(137), atol=1e-10)


@pytest.mark.parametrize("lam,prec,nt,nwb", [(1e4, "low", 48, 49), (1e5, "low", 61, 61),
                                             (1e4, "high", 104, 105), (1e4, "medium", 74, 75),
                                             (1e3, "low", 34, 35)])
def test_grid_sizes(lam, prec, nt, nwb):
    ft = IAFT(1000.0, lam / 1000.0, prec)
    assert (ft.nt_f, ft.nw_b) == (nt, nwb)
    np.testing.assert_allclose(ft.Ttw_ff @ ft.Twt_ff, np.eye(nt), atol=1e-9)
    np.testing.assert_allclose(ft.Ttw_bb @ ft.Twt_bb, np.eye(nt), atol=1e-9)
    # tau meshes are particle-hole symmetric (thc_gw.cpp:56-66)
    x = ft.tau_mesh_x
    assert np.all(np.abs(np.abs(x) - np.abs(x[::-1])) <= 1e-6)


@pytest.mark.parametrize("prec", ["low", "high"])
def test_product_ph_matrices_match_oracle(prec):
    o = IAFT(1000.0, 10.0, prec)
    p = ProductIAFT(1000.0, 10.0, prec)
    assert p.check_ph_symmetric()
    np.testing.assert_array_equal(p.Twt_pos(), o.Twt_pos())
    np.testing.assert_array_equal(p.Ttw_pos(), o.Ttw_pos())
    np.testing.assert_array_equal(p.Ttw_bb, o.Ttw_bb)


def test_lambda_rounding():
    from oracle.thc_oracle import determine_lambda
    assert determine_lambda(1200) == 1e4 and determine_lambda(100) == 100
    assert determine_lambda(1e6) == 1e6 and determine_lambda(2e6) == -1
