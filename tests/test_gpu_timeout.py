"""Bounded device waits: a tensor-core kernel whose wait runs out returns an error status.

Every wait of the tensor-core GEMMs (producers on a free stage, the MMA lane on a filled
stage and on a free accumulator, the epilogue on a finished accumulator) is bounded.  With
the limit set to a few nanoseconds the waits run out: the kernel sets its error flag, lets
the tensor-core work it issued retire, frees its tensor memory and returns, the call reports
COQUI_B200_ETIMEDOUT, and after the default limit is restored the same context gives the
same result as before.  Both kernel forms (one tile per CTA, persistent) are exercised; no
fault, trap or hang is involved.
"""
import numpy as np
import pytest

from coqui_b200 import capi
from coqui_b200.iaft import IAFT
from coqui_b200.synthetic import make_system

pytestmark = pytest.mark.gpu

ETIMEDOUT = -7


@pytest.fixture(scope="module")
def case():
    s = make_system(2, 64, 24, 256, seed=31)
    ft = IAFT(1000.0, 10.0, "low")
    return s, ft, s.G0(ft)[:4]


# single-stage tiles (the producers must wait for the MMA lane at every K block) in the
# one-tile-per-CTA form and in the persistent form
@pytest.mark.parametrize("cfg", [0, 6], ids=["per_tile", "persistent"])
def test_wait_runs_out_and_context_recovers(case, cfg):
    s, ft, G = case
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=capi.MIXED)
    try:
        c.set_ir(ft)
        c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
        c.set_thc(s.X, s.V)
        capi.set_tile_config(cfg)
        ref = c.primary_to_aux(G)
        capi.set_wait_limit_ns(1)
        with pytest.raises(capi.CoquiB200Error) as err:
            c.primary_to_aux(G)
        assert err.value.code == ETIMEDOUT
        capi.set_wait_limit_ns(0)
        again = c.primary_to_aux(G)
        assert np.array_equal(again, ref)
    finally:
        capi.set_wait_limit_ns(0)
        capi.set_tile_config(-1)
        c.close()
