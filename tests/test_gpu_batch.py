"""Uneven batch of Gamma-only molecules with fused launches against the FP64 oracle and
against the single-system context run per molecule (mixed precision, tolerance 1e-6)."""
import numpy as np
import pytest

from coqui_b200 import capi
from coqui_b200.iaft import IAFT
from coqui_b200.synthetic import make_system
from oracle import thc_oracle as O

pytestmark = pytest.mark.gpu

# (orbitals, interpolating points): one to three tensor-core inverse levels above Np = 128
SIZES = [(8, 48), (12, 72), (6, 36), (16, 150), (10, 260), (20, 540)]


@pytest.fixture(scope="module")
def molecules():
    ft = IAFT(500.0, 20.0, "low")
    oft = O.IAFT(500.0, 20.0, "low")
    mols = []
    for i, (nb, Np) in enumerate(SIZES):
        s = make_system(1, nb, nb // 2, Np, beta=500.0, seed=40 + i, gamma_only=True)
        G = s.G0(oft)
        dW, _, _ = O.update_w(G, s.X, s.V, oft, s.kpts, s.lattv, s.kp_grid)
        Sigma = O.eval_Sigma_all_Rspace(G, dW, s.X, s.kpts, s.lattv, s.kp_grid)
        mols.append(dict(s=s, G=G, Sigma=Sigma))
    return ft, mols


def test_fused_batch_matches_oracle_and_per_molecule_contexts(molecules):
    ft, mols = molecules
    b = capi.Batch([m["s"].nb for m in mols], [m["s"].Np for m in mols], ft.nt_f, ft.nw_b)
    b.set_ir(ft)
    for i, m in enumerate(mols):
        b.set_thc(i, m["s"].X[0, 0], m["s"].V[0])
    out = b.gw_iteration([m["G"][:, 0, 0] for m in mols])
    for m, S in zip(mols, out):
        assert np.abs(S - m["Sigma"][:, 0, 0]).max() < 1e-6
        s = m["s"]
        c = capi.Context(1, s.nb, s.Np, ft.nt_f, ft.nw_b, (1, 1, 1), mode=capi.MIXED)
        c.set_ir(ft)
        c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
        c.set_thc(s.X, s.V)
        S1, _ = c.gw_iteration(m["G"])
        assert np.abs(S - S1[:, 0, 0]).max() < 1e-6
        c.close()
    # a second iteration on the same buffers gives the same result
    out2 = b.gw_iteration([m["G"][:, 0, 0] for m in mols])
    assert max(np.abs(a - c).max() for a, c in zip(out, out2)) < 1e-12
    b.close()


def test_batch_rejects_missing_set_up():
    ft = IAFT(500.0, 20.0, "low")
    b = capi.Batch([4, 5], [16, 20], ft.nt_f, ft.nw_b)
    with pytest.raises(capi.CoquiB200Error) as e:
        b.gw_iteration([np.zeros((ft.nt_f, 4, 4)), np.zeros((ft.nt_f, 5, 5))])
    assert e.value.code == -1
    b.close()


def test_page_locked_sigma_has_landed_when_the_call_returns(molecules):
    """With page-locked output buffers the device-to-host copies return at once: the call
    itself must wait for them, so Sigma read right after it equals Sigma copied to pageable
    buffers."""
    import torch
    ft, mols = molecules
    b = capi.Batch([m["s"].nb for m in mols], [m["s"].Np for m in mols], ft.nt_f, ft.nw_b)
    b.set_ir(ft)
    for i, m in enumerate(mols):
        b.set_thc(i, m["s"].X[0, 0], m["s"].V[0])
    Gs = [m["G"][:, 0, 0] for m in mols]
    ref = b.gw_iteration(Gs)
    pinned = []
    for S in ref:
        h = torch.empty(S.shape, dtype=torch.complex128, pin_memory=True).numpy()
        h[...] = np.nan
        pinned.append(h)
    out = b.gw_iteration(Gs, pinned)
    for S, P in zip(ref, out):
        assert np.array_equal(S, P)
    b.close()
