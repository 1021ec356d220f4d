"""THC ERI file reader (thc_reader_t::read, thc_reader_t.hpp:507-574): files in the
reference's "bdft" layout (dataset names and shapes of thc_reader_t.hpp:233-256 and
thc.cpp:362-378, complex values as a trailing (re, im) dimension) are read into the arrays the
device path takes, and inconsistent files are refused with the reference's checks.

The reference ships no THC ERI file (its ISDF builder writes them at run time), so the files
here are written by tests/h5write.py in that layout; the HDF5 decoder itself is also checked
on the reference's own HDF5 files (the IR tables and Green's-function fixtures,
tests/test_oracle_golden.py and tests/golden/convert_ir_tables.py).
"""
import numpy as np
import pytest

from coqui_b200.synthetic import make_system
from coqui_b200.thc_file import read_thc_file
from tests.h5write import write_h5


def thc_datasets(s, **over):
    nk, Np, nb = s.nk, s.Np, s.nb
    d = {
        "Np": np.int32(Np), "number_of_bands": np.int32(nb),
        "X_orbital_range": np.array([0, nb], np.int32), "Y_orbital_range": np.array([0, nb], np.int32),
        "kpts": s.kpts, "qpts": s.kpts, "nkpts_ibz": np.int32(nk), "nqpts_ibz": np.int32(nk),
        "collocation_matrix": s.X, "interpolating_points": np.arange(Np, dtype=np.int64),
        "interpolating_vectors_G0": s.chi_bar * 2.0, "dual_interpolating_vectors_G0": s.chi_bar,
        "coulomb_matrix": s.V,
    }
    d.update(over)
    return d


@pytest.fixture(scope="module")
def system():
    return make_system(2, 8, 4, 24, seed=3)


def test_round_trip(tmp_path, system):
    s = system
    p = str(tmp_path / "thc.h5")
    write_h5(p, thc_datasets(s))
    t = read_thc_file(p, s.lattv, s.kp_grid, madelung=0.25)
    assert np.array_equal(t.X, s.X) and np.array_equal(t.V, s.V)
    assert np.array_equal(t.kpts, s.kpts) and np.array_equal(t.chi_bar, s.chi_bar)
    assert np.array_equal(t.chi_head, 2.0 * s.chi_bar[0]) and t.madelung == 0.25
    assert (t.Np, t.nbnd, t.nkpts, t.kp_grid) == (s.Np, s.nb, s.nk, s.kp_grid)


@pytest.mark.parametrize("bad,msg", [
    (dict(interpolating_points=np.arange(5)), "rp.shape"),
    (dict(X_orbital_range=np.array([0, 99], np.int32)), "X_orbital_range"),
    (dict(nqpts_ibz=np.int32(3)), "bz maps"),
    (dict(Y_orbital_range=np.array([0, 4], np.int32)), "Y collocation"),
])
def test_inconsistent_files_are_refused(tmp_path, system, bad, msg):
    s = system
    p = str(tmp_path / "bad.h5")
    write_h5(p, thc_datasets(s, **bad))
    with pytest.raises(ValueError, match=msg):
        read_thc_file(p, s.lattv, s.kp_grid)


def test_missing_dataset_is_refused(tmp_path, system):
    s = system
    d = thc_datasets(s)
    del d["coulomb_matrix"]
    p = str(tmp_path / "short.h5")
    write_h5(p, d)
    with pytest.raises(ValueError, match="missing"):
        read_thc_file(p, s.lattv, s.kp_grid)


@pytest.mark.gpu
def test_solvers_from_a_thc_file_match_the_oracle(tmp_path):
    """update_w + evaluate through the solver mirror on THC data read from a file."""
    from coqui_b200 import solvers
    from coqui_b200.iaft import IAFT
    from oracle import thc_oracle as O
    s = make_system(2, 16, 8, 64, seed=9)
    p = str(tmp_path / "thc.h5")
    write_h5(p, thc_datasets(s))
    thc = read_thc_file(p, s.lattv, s.kp_grid)
    ft, oft = IAFT(1000.0, 10.0, "low"), O.IAFT(1000.0, 10.0, "low")
    G = s.G0(oft)
    mb = solvers.MBState(sG_tskij=G)
    solvers.scr_coulomb_t(ft).update_w(mb, thc)
    solvers.gw_t(ft).evaluate(mb, thc)
    dW, _, _ = O.update_w(G, s.X, s.V, oft, s.kpts, s.lattv, s.kp_grid, s.chi_bar)
    S_ref = O.eval_Sigma_all_Rspace(G, dW, s.X, s.kpts, s.lattv, s.kp_grid)
    assert np.abs(mb.sSigma_tskij - S_ref).max() < 1e-6


def sym_datasets(d):
    """A symmetric mean field's file: X on every k-point and kpts in the mean field's order
    (IBZ first), V and the dual heads on the IBZ q-points only."""
    sym = d["sym"]
    nk, nqi = sym["nk"], sym["nq_ibz"]
    X = d["X"]
    Np, nb = X.shape[2], X.shape[3]
    return {
        "Np": np.int32(Np), "number_of_bands": np.int32(nb),
        "X_orbital_range": np.array([0, nb], np.int32), "Y_orbital_range": np.array([0, nb], np.int32),
        "kpts": d["kpts"], "qpts": d["kpts"], "nkpts_ibz": np.int32(sym["nk_ibz"]),
        "nqpts_ibz": np.int32(nqi), "collocation_matrix": X,
        "interpolating_points": np.arange(Np, dtype=np.int64),
        "interpolating_vectors_G0": d["chi_bar"][:1] * 2.0,
        "dual_interpolating_vectors_G0": d["chi_bar"][:nqi], "coulomb_matrix": d["V"][:nqi],
    }


def test_symmetry_reduced_file_with_the_bz_maps(tmp_path):
    from coqui_b200.iaft import IAFT
    from coqui_b200.symmetry import symmetric_system
    d = symmetric_system("swap", (4, 4, 1), 6, 12, IAFT(1000.0, 10.0, "low"))
    sym = d["sym"]
    p = str(tmp_path / "thc_sym.h5")
    write_h5(p, sym_datasets(d))
    with pytest.raises(ValueError, match="bz maps"):
        read_thc_file(p, d["lattv"], d["grid"])
    t = read_thc_file(p, d["lattv"], d["grid"], bz=sym, bz_rotations=d["D"])
    assert np.array_equal(t.X, d["X_lex"]) and np.allclose(t.kpts, d["kpts_lex"])
    ql = d["lex"][:sym["nq_ibz"]]
    assert np.array_equal(t.V[ql], d["V"][:sym["nq_ibz"]])
    assert np.array_equal(t.chi_bar[ql], d["chi_bar"][:sym["nq_ibz"]])
    assert t.bz is sym and t.bz_rotations is d["D"]


@pytest.mark.gpu
def test_solvers_from_a_symmetry_reduced_file_match_the_kspace_oracle(tmp_path):
    """A symmetric mean field's file read with its bz maps runs the k-space routes."""
    from coqui_b200 import capi, solvers
    from coqui_b200.iaft import IAFT
    from coqui_b200.symmetry import symmetric_system
    from oracle import sym_oracle as SO
    from oracle import thc_oracle as O
    ft, oft = IAFT(1000.0, 10.0, "low"), O.IAFT(1000.0, 10.0, "low")
    d = symmetric_system("swap", (4, 4, 1), 8, 24, oft)
    sym = d["sym"]
    p = str(tmp_path / "thc_sym.h5")
    write_h5(p, sym_datasets(d))
    thc = read_thc_file(p, d["lattv"], d["grid"], bz=sym, bz_rotations=d["D"])
    mb = solvers.MBState(sG_tskij=d["G_ibz"])
    try:
        solvers.scr_coulomb_t(ft, mode=capi.FP64).update_w(mb, thc)
        solvers.gw_t(ft, mode=capi.FP64).evaluate(mb, thc)
    finally:
        solvers.clear_contexts()
    dW = SO.update_w_kspace(d["G_ibz"], d["X"], d["V"], oft, sym)
    S_ref = SO.eval_Sigma_all_kspace(d["G_ibz"], dW, d["X"], sym, d["D"])
    assert np.abs(mb.dW_qtPQ - dW).max() < 1e-10
    assert np.abs(mb.sSigma_tskij - S_ref).max() < 1e-10
