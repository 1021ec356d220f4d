"""Symmetry-reduced k-space oracle (CPU): the bz_symm lists, and the reference's k-space
polarizability, screened interaction, self-energy and RPA energy on the IBZ against the
full-BZ R-space restatement on symmetric inputs.

Identities of the two reference routes (exact for any G, V with V(-q) = conj V(q)):
Pi_k(q) = Pi_R(-q)^T, W_k(q) = W_R(-q)^T; Sigma_k from W_R at the IBZ q-points equals
Sigma_R at the IBZ k-points; E_c agrees.  The mirror model has a nontrivial rotation D on the
mirror line, so the D^H Sigma D step of thc_gw.icc:302-310 is exercised."""
import numpy as np
import pytest

from oracle import sym_oracle as SO
from oracle import thc_oracle as O
from coqui_b200 import symmetry as SY
from coqui_b200.symmetry import symmetric_system as make_sym_system

CASES = [("trev", (4, 1, 1)), ("trev", (3, 3, 1)), ("swap", (3, 3, 1)), ("swap", (4, 4, 1))]


@pytest.fixture(scope="module")
def ft():
    return O.IAFT(1000.0, 10.0, "low")


@pytest.mark.parametrize("kind,grid", CASES, ids=[f"{k}-{g[0]}{g[1]}{g[2]}" for k, g in CASES])
def test_kspace_equals_full_bz(ft, kind, grid):
    d = make_sym_system(kind, grid, 6, 12, ft)
    sym = d["sym"]
    ql = d["lex"][:sym["nq_ibz"]]
    mql = d["lex"][sym["qminus"][:sym["nq_ibz"]]]
    kl = d["lex"][:sym["nk_ibz"]]
    args = (d["kpts_lex"], d["lattv"], d["grid"])
    Pi_R = O.eval_Pi_rpa_Rspace(d["G_lex"], d["X_lex"], *args)
    Pi_k = SO.eval_Pi_rpa_kspace(d["G_ibz"], d["X"], sym)
    assert np.abs(Pi_k - np.swapaxes(Pi_R[:, mql], -1, -2)).max() < 1e-13
    dW_R, _, _ = O.update_w(d["G_lex"], d["X_lex"], d["V_lex"], ft, *args)
    dW_k = SO.update_w_kspace(d["G_ibz"], d["X"], d["V"], ft, sym)
    assert np.abs(dW_k - np.swapaxes(dW_R[mql], -1, -2)).max() < 1e-12
    S_R = O.eval_Sigma_all_Rspace(d["G_lex"], dW_R, d["X_lex"], *args)
    S_k = SO.eval_Sigma_all_kspace(d["G_ibz"], dW_R[ql], d["X"], sym, d["D"])
    assert np.abs(S_k - S_R[:, :, kl]).max() < 1e-12
    e_R = O.rpa_energy(d["G_lex"], d["X_lex"], d["V_lex"], ft, *args)
    e_k = SO.rpa_energy_kspace(d["G_ibz"], d["X"], d["V"], ft, sym)
    assert abs(e_k - e_R) < 1e-12
    assert abs(e_R) > 1e-3


def test_time_reversal_kspace_sigma_is_the_full_bz_sigma(ft):
    # with time reversal the k-space W is the R-space W itself, so the whole k-space chain
    # reproduces the full-BZ self-energy
    d = make_sym_system("trev", (3, 3, 1), 6, 12, ft)
    sym = d["sym"]
    args = (d["kpts_lex"], d["lattv"], d["grid"])
    dW_R, _, _ = O.update_w(d["G_lex"], d["X_lex"], d["V_lex"], ft, *args)
    S_R = O.eval_Sigma_all_Rspace(d["G_lex"], dW_R, d["X_lex"], *args)
    dW_k = SO.update_w_kspace(d["G_ibz"], d["X"], d["V"], ft, sym)
    S_k = SO.eval_Sigma_all_kspace(d["G_ibz"], dW_k, d["X"], sym, d["D"])
    assert np.abs(S_k - S_R[:, :, d["lex"][:sym["nk_ibz"]]]).max() < 1e-12


SYM_LISTS = [("trev", (3, 3, 1), True), ("swap", (4, 4, 1), False), ("both", (4, 4, 1), True),
             ("both", (3, 3, 2), True)]


def _ops(kind):
    return [np.eye(3, dtype=int)] + ([] if kind == "trev" else [SY.SWAP])


@pytest.mark.parametrize("kind,grid,use_trev", SYM_LISTS)
def test_library_lists_equal_the_oracle_restatement(kind, grid, use_trev):
    a = SY.bz_symmetry(grid, _ops(kind), use_trev)
    b = SO.build_bz_symmetry(grid, _ops(kind), use_trev)
    for key in b:
        assert np.array_equal(np.asarray(a[key]), np.asarray(b[key])), key


@pytest.mark.parametrize("kind,grid,use_trev", SYM_LISTS)
def test_bz_symmetry_lists(kind, grid, use_trev):
    ops = _ops(kind)
    s = SY.bz_symmetry(grid, ops, use_trev)
    nk, nki = s["nk"], s["nk_ibz"]
    assert nk == int(np.prod(grid)) and sorted(s["lex"]) == list(range(nk))
    # IBZ first and mapped to themselves; time-reversal images last, paired with -k
    assert list(s["kp_to_ibz"][:nki]) == list(range(nki)) and not s["kp_trev"][:nki].any()
    tr = np.flatnonzero(s["kp_trev"])
    if tr.size:
        assert tr.min() >= nk - tr.size
    g = np.array(grid)
    for i in tr:
        p = s["kp_trev_pair"][i]
        assert not s["kp_trev"][p] and np.all((s["kc"][i] + s["kc"][p]) % g == 0)
    # every k is an image of its IBZ point under its operation (and -1 when kp_trev)
    for i in range(nk):
        M = ops[s["kp_symm"][i]]
        img = (M @ s["kc"][s["kp_to_ibz"][i]]) * (-1 if s["kp_trev"][i] else 1) % g
        assert np.all(img == s["kc"][i])
    # Qs rows partition the q-points; ks_to_k is the inverse operation on k
    qs = np.concatenate([s["Qs"][i, :s["nq_per_s"][i]] for i in range(len(s["qsymms"]))])
    assert sorted(qs) == list(range(nk))
    for i, sy in enumerate(s["qsymms"]):
        Rt = np.rint(np.linalg.inv(ops[sy])).astype(int)
        for k in range(nk):
            assert np.all((Rt @ s["kc"][k]) % g == s["kc"][s["ks_to_k"][i, k]])
    # qk_to_k2 = k - q, qminus = -q
    for q in range(nk):
        assert np.all((s["kc"][q] + s["kc"][s["qminus"][q]]) % g == 0)
        for k in range(nk):
            assert np.all((s["kc"][k] - s["kc"][q] - s["kc"][s["qk_to_k2"][q, k]]) % g == 0)
