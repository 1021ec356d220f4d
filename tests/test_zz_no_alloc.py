"""The allocation-free projection entry point against the regular one.

coqui_b200_primary_to_aux_noalloc serves callers that hold their own device buffers and may
not allocate device memory (their memory comes from their own pool, or they run under a
fixed device-memory budget).  It runs the same tensor-core projection as
coqui_b200_primary_to_aux but keeps every intermediate in the library's static 32 MiB
device array.  This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import numpy as np
import pytest

from coqui_b200 import capi
from coqui_b200.iaft import IAFT
from coqui_b200.synthetic import make_system

pytestmark = pytest.mark.gpu

TOL = 1e-6  # the mixed-precision tolerance of the other parity tests


def test_noalloc_projection_matches_context_projection_twice():
    import torch

    s = make_system(2, 16, 8, 64, seed=5)
    ft = IAFT(1000.0, 10.0, "low")
    G = s.G0(ft)
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=capi.MIXED)
    c.set_ir(ft)
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    taus = [3, ft.nt_f - 4]
    ref = c.primary_to_aux(G[taus])  # (2, 1, nk, Np, Np) complex128, existing entry point

    dev = torch.device("cuda", 0)
    X_d = torch.from_numpy(np.ascontiguousarray(s.X[0])).to(dev)
    out = torch.empty((s.nk, s.Np, s.Np), dtype=torch.complex64, device=dev)
    free_after = []
    for i, t in enumerate(taus):  # two calls in a row share the static scratch array
        G_d = torch.from_numpy(np.ascontiguousarray(G[t, 0])).to(dev)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        capi.primary_to_aux_noalloc(X_d.data_ptr(), G_d.data_ptr(), out.data_ptr(), s.nk, s.Np,
                                    s.nb)
        torch.cuda.synchronize()
        free_after.append((free_before, torch.cuda.mem_get_info(dev)[0]))
        got = out.cpu().numpy().astype(np.complex128)
        assert float(np.abs(got - ref[i, 0]).max()) < TOL
    # the first call may load the library's device code (and with it the static array);
    # from then on a call leaves the device's free memory exactly as it found it
    assert free_after[1][0] == free_after[1][1]
    c.close()


def test_noalloc_rejects_oversized_problems_and_host_pointers():
    import torch

    with pytest.raises(capi.CoquiB200Error) as e:  # 64 x 1024 x 96: ~200 MB of scratch
        capi.primary_to_aux_noalloc(1, 1, 1, 64, 1024, 96)
    assert e.value.code == -1 and "static limit" in str(e.value)
    host = np.zeros(16, np.complex128)
    dev = torch.zeros(64, dtype=torch.complex128, device="cuda")
    with pytest.raises(capi.CoquiB200Error) as e:
        capi.primary_to_aux_noalloc(host.ctypes.data, dev.data_ptr(), dev.data_ptr(), 1, 2, 2)
    assert e.value.code == -1 and "device pointers" in str(e.value)
