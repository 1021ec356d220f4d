"""GPU parity of the pipelined paths: G arriving in tau chunks from page-locked memory, Sigma
leaving chunk by chunk, and the projected-G cache shared by the polarizability and the
self-energy of one G.

A 4x4x4 grid gives 64 (tau, k) problems per tau slice, so the Sigma/Pi loops run in several
chunks of 4 tau pairs; Lambda = 1e5 gives an odd nt (61) whose middle slice is its own
particle-hole partner.  Tolerances as in test_gpu_parity.
"""
import numpy as np
import pytest

from coqui_b200 import capi
from coqui_b200.iaft import IAFT as ProductIAFT
from coqui_b200.synthetic import make_system
from oracle import thc_oracle as O

pytestmark = pytest.mark.gpu

MODES = [(capi.FP64, 1e-10), (capi.MIXED, 1e-6)]
MODE_IDS = ["fp64", "mixed"]


def maxabs(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max())


@pytest.fixture(scope="module", params=[1e4, 1e5], ids=["nt48", "nt61"])
def case(request):
    lam = request.param
    s = make_system(4, 8, 4, 32, seed=21)
    ft = O.IAFT(1000.0, lam / 1000.0, "low")
    G = s.G0(ft)
    dW, head, _ = O.update_w(G, s.X, s.V, ft, s.kpts, s.lattv, s.kp_grid, s.chi_bar)
    Sigma = O.eval_Sigma_all_Rspace(G, dW, s.X, s.kpts, s.lattv, s.kp_grid)
    e_rpa = O.rpa_energy(G, s.X, s.V, ft, s.kpts, s.lattv, s.kp_grid)
    return dict(s=s, ft=ft, pft=ProductIAFT(1000.0, lam / 1000.0, "low"), G=G, dW=dW,
                head=head, Sigma=Sigma, e_rpa=e_rpa)


def make_ctx(case, mode):
    s, ft = case["s"], case["ft"]
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=mode)
    c.set_ir(case["pft"])
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    return c


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_pinned_buffers_take_the_chunked_path(case, mode, tol):
    import torch

    c = make_ctx(case, mode)
    G_pinned = torch.from_numpy(np.ascontiguousarray(case["G"])).pin_memory()
    S_pinned = torch.zeros(G_pinned.shape, dtype=torch.complex128).pin_memory()
    c.gw_iteration(G_pinned.numpy(), sigma_out=S_pinned.numpy())
    assert maxabs(S_pinned.numpy(), case["Sigma"]) < tol
    # pageable buffers (one copy each) give the same numbers
    S_pageable, _ = c.gw_iteration(np.ascontiguousarray(case["G"]))
    assert maxabs(S_pageable, S_pinned.numpy()) < 1e-12
    # eval_sigma with a page-locked G: chunked upload, no cache, chunked download
    S_pinned.zero_()
    c.eval_sigma(G_pinned.numpy(), out=S_pinned.numpy())
    assert maxabs(S_pinned.numpy(), case["Sigma"]) < tol
    c.close()


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_sigma_after_update_w_uses_the_same_g_only(case, mode, tol):
    c = make_ctx(case, mode)
    c.update_w(case["G"])
    # resident G: the projections cached by update_w are reused
    assert maxabs(c.eval_sigma(None), case["Sigma"]) < tol
    # a different G after update_w must not see the cached projections (Sigma is linear in G)
    c.update_w(case["G"])
    assert maxabs(c.eval_sigma(0.5 * case["G"]), 0.5 * case["Sigma"]) < tol
    # the cache was overwritten in place by the previous Sigma: recomputed from resident G
    assert maxabs(c.eval_sigma(None), 0.5 * case["Sigma"]) < tol
    c.close()


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_resident_g_survives_building_block_calls(case, mode, tol):
    c = make_ctx(case, mode)
    c.update_w(case["G"])
    # primary_to_aux stages its own input: the resident G and its cached projections stay valid
    out = c.primary_to_aux(case["G"][:2] * 3.0)
    assert maxabs(out, O.primary_to_aux(case["G"][:2] * 3.0, case["s"].X[None])) < tol * 3
    assert maxabs(c.eval_sigma(None), case["Sigma"]) < tol
    assert abs(c.rpa_energy(None) - case["e_rpa"]) < tol
    c.close()


def test_resident_iteration_graph_matches_direct_launches(case):
    """gw_iteration with a resident G and no host outputs runs as a captured CUDA graph (the
    first of consecutive calls captures, the next ones replay); W and Sigma are those of the
    directly launched path."""
    c = make_ctx(case, capi.MIXED)
    S_direct, _ = c.gw_iteration(case["G"])
    n0 = c.kernel_launches()
    c.gw_iteration(None, want_sigma=False)  # capture + launch
    n1 = c.kernel_launches()
    c.gw_iteration(None, want_sigma=False)  # replay
    n2 = c.kernel_launches()
    assert n1 - n0 == n2 - n1 > 0
    assert [name for name, _ in c.timings()] == ["GW_ITERATION_GRAPH"]
    # W from the replayed graph feeds Sigma: identical to the direct path
    S_graph = c.eval_sigma(None)
    assert np.array_equal(S_graph, S_direct)
    c.close()


def test_graph_capture_of_tiled_factorisation_and_tensor_core_inverse():
    """Np = 300 with one q: a few large Dyson problems take the tiled factorisation and the
    tensor-core inverse levels; both are captured in the resident-G graph and replay to the
    directly launched result."""
    s = make_system(1, 16, 8, 300, seed=7, gamma_only=True)
    ft = O.IAFT(1000.0, 10.0, "low")
    G = s.G0(ft)
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=capi.MIXED)
    c.set_ir(ProductIAFT(1000.0, 10.0, "low"))
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    S_direct, _ = c.gw_iteration(G)
    c.gw_iteration(None, want_sigma=False)  # capture + launch
    c.gw_iteration(None, want_sigma=False)  # replay
    assert [name for name, _ in c.timings()] == ["GW_ITERATION_GRAPH"]
    assert np.array_equal(c.eval_sigma(None), S_direct)
    c.close()


def test_pinned_host_buffer_iteration_runs_as_a_graph(case):
    """gw_iteration with page-locked G in and Sigma out runs as one graph with its copies:
    replayed for the same buffers, captured again for new ones, always the directly launched
    result (pageable buffers take the direct path)."""
    import torch
    c = make_ctx(case, capi.MIXED)
    S_direct, _ = c.gw_iteration(np.ascontiguousarray(case["G"]))  # pageable: direct path
    assert "GW_ITERATION_GRAPH" not in [name for name, _ in c.timings()]
    outs = []
    for _ in range(2):
        G_p = torch.from_numpy(np.ascontiguousarray(case["G"])).pin_memory()
        S_p = torch.zeros(G_p.shape, dtype=torch.complex128).pin_memory()
        for _ in range(2):  # capture + launch, then replay
            S_p.zero_()
            c.gw_iteration(G_p.numpy(), sigma_out=S_p.numpy())
            assert [name for name, _ in c.timings()] == ["GW_ITERATION_GRAPH"]
            outs.append(S_p.numpy().copy())
    for S in outs:
        assert np.array_equal(S, S_direct)
    c.close()


def test_rpa_energy_graph_matches_direct_launches(case):
    """In mixed mode the RPA energy of a resident or page-locked G runs as a CUDA graph
    (captured on the first of consecutive calls with the same G argument, replayed by the
    next): the same energy as the directly launched call on a pageable G."""
    import torch

    c = make_ctx(case, capi.MIXED)
    e0 = c.rpa_energy(np.ascontiguousarray(case["G"]))  # pageable: launched directly
    assert abs(e0 - case["e_rpa"]) < 1e-6
    G_pinned = torch.from_numpy(np.ascontiguousarray(case["G"])).pin_memory().numpy()
    energies = [c.rpa_energy(G_pinned), c.rpa_energy(G_pinned),  # capture (copy inside), replay
                c.rpa_energy(None), c.rpa_energy(None)]          # resident G: capture, replay
    for e in energies:
        assert abs(e - e0) < 1e-12, (e, e0)
    names = [n for n, _ in c.timings()]
    assert names == ["RPA_GRAPH"], names
    # a GW iteration between two RPA calls: the RPA graph is captured again, same energy
    c.gw_iteration(None, want_sigma=False)
    assert abs(c.rpa_energy(None) - e0) < 1e-12
    c.close()


@pytest.mark.parametrize("mode,tol", MODES, ids=MODE_IDS)
def test_partial_projection_cache(case, mode, tol):
    """The projected-G cache holding every slice, only the first tau chunk (slices [0, 4) and
    [nt - 4, nt)), or nothing: the self-energy is the same, and the counted projections are the
    polarizability's 2 nth per k plus the slices the self-energy projects again."""
    s, ft = case["s"], case["ft"]
    c = make_ctx(case, mode)
    G = np.ascontiguousarray(case["G"])
    nt, nk = ft.nt_f, s.nk
    nth = (nt + 1) // 2
    chunk = min(nth, max(4, -(-256 // nk)))
    slab = nk * s.Np ** 2 * (16 if mode == capi.FP64 else 8)
    res = {}
    for name, limit, again in (("all", -1, 0), ("one_chunk", 2 * chunk * slab, nt - 2 * chunk),
                               ("none", 0, nt)):
        c.set_gcache_limit(limit)
        c.set_profiling(True)
        S, _ = c.gw_iteration(G)
        units = c.kernel_units()
        c.set_profiling(False)
        res[name] = S
        assert units["proj_p2a"] == (2 * nth + again) * nk, name
    assert maxabs(res["all"], case["Sigma"]) < tol
    assert maxabs(res["one_chunk"], res["all"]) < 1e-12
    assert maxabs(res["none"], res["all"]) < 1e-12
    c.set_gcache_limit(-1)
    with pytest.raises(capi.CoquiB200Error):
        c.set_gcache_limit(-2)
