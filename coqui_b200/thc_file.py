"""Reader of CoQui's precomputed THC ERI file (``thc_reader_t::read``,
src/methods/ERI/thc_reader_t.hpp:507-574; written by the same class at :233-256 and by
``thc::save``, src/methods/ERI/thc.cpp:362-378, "bdft" format).

The file is HDF5 through TRIQS h5 (decoded by :mod:`coqui_b200.h5lite`; complex arrays carry a
trailing (re, im) dimension).  Datasets of the root group:

* ``Np``, ``number_of_bands`` (scalars), ``X_orbital_range`` / ``Y_orbital_range`` ([first,
  last) band ranges), ``kpts``, ``qpts``, ``nkpts_ibz``, ``nqpts_ibz``;
* ``collocation_matrix`` (ns*npol, nkpts, Np, nbnd_X) and, for a different Y range,
  ``Y_collocation_matrix``;
* ``interpolating_points`` (Np), ``interpolating_vectors_G0`` / ``dual_interpolating_vectors_G0``
  (the q -> 0 heads of the interpolating vectors and of their duals, (nq, Np));
* ``coulomb_matrix`` (nqpts_ibz, Np, Np): the reference's in-memory Z (already multiplied by
  nkpts before it was written), which is V here.

The lattice vectors and the k-grid come from the mean field, as in the reference.  Checks and
their messages follow ``thc_reader_t::read``; X and Y must cover the same band range.

A file of a symmetric mean field (nkpts_ibz or nqpts_ibz below nkpts) stores X on every
k-point in the mean field's order (IBZ first) and V only on the IBZ q-points.  It is read with
the mean field's bz maps (``bz``, as :func:`coqui_b200.symmetry.bz_symmetry` lays them out,
and the rotations ``bz_rotations``): X, kpts and the heads are put in lexicographic grid
order, and every 1st-BZ q-point's V slot holds the matrix of its IBZ point (the k-space routes
read only the IBZ slots; the full-BZ routes must not be used on such data, and the solver
mirror's Hartree-Fock refuses it).  The returned THCData carries the maps, so the solver
mirror takes the reference's k-space routes.
"""
from __future__ import annotations

import numpy as np

from . import h5lite
from .solvers import THCData


def _scalar(a):
    return int(np.asarray(a).reshape(-1)[0])


def read_thc_file(path: str, lattv, kp_grid, madelung: float = 0.0, bz=None,
                  bz_rotations=None) -> THCData:
    """THCData from a THC ERI file; lattv (3, 3) and kp_grid (3,) are the mean field's, and bz
    / bz_rotations its symmetry maps (needed for a symmetry-reduced file)."""
    d = h5lite.read_h5(path)
    need = ("Np", "X_orbital_range", "Y_orbital_range", "interpolating_points",
            "collocation_matrix", "coulomb_matrix")
    missing = [n for n in need if n not in d]
    if missing:
        raise ValueError(f"thc_reader_t::read(): missing datasets {missing}")
    Np = _scalar(d["Np"])
    X = h5lite.as_complex(d["collocation_matrix"])
    if X.ndim != 4:
        raise ValueError("thc_reader_t::read(): collocation_matrix is not (ns*npol, nk, Np, nbnd)")
    nbnd = _scalar(d["number_of_bands"]) if "number_of_bands" in d else X.shape[3]
    xr = [int(v) for v in np.asarray(d["X_orbital_range"]).reshape(-1)]
    yr = [int(v) for v in np.asarray(d["Y_orbital_range"]).reshape(-1)]
    for name, r in (("X", xr), ("Y", yr)):
        if not (len(r) == 2 and r[0] >= 0 and r[1] <= nbnd):
            raise ValueError(f"thc_reader::read(): Invalid {name}_orbital_range.")
    rp = np.asarray(d["interpolating_points"]).reshape(-1)
    if rp.shape[0] != Np:
        raise ValueError("thc_reader_t::build: rp.shape() != Np. Inconsistent dimensions from "
                         "the precomputed THC-ERI.")
    if X.shape[2] != Np or X.shape[3] != xr[1] - xr[0]:
        raise ValueError("thc_reader_t::read(): collocation_matrix shape does not match Np and "
                         "X_orbital_range")
    if xr != yr or "Y_collocation_matrix" in d:
        raise ValueError("a Y collocation matrix over another band range is not supported")
    V = h5lite.as_complex(d["coulomb_matrix"])
    nk = X.shape[1]
    if V.shape != (V.shape[0], Np, Np):
        raise ValueError("thc_reader_t::read(): coulomb_matrix is not (nqpts_ibz, Np, Np)")
    nk_ibz = _scalar(d["nkpts_ibz"]) if "nkpts_ibz" in d else nk
    nq_ibz = _scalar(d["nqpts_ibz"]) if "nqpts_ibz" in d else V.shape[0]
    reduced = nk_ibz != nk or nq_ibz != nk or V.shape[0] != nk
    if reduced and bz is None:
        raise ValueError("symmetry-reduced file (nkpts_ibz or nqpts_ibz below nkpts): pass the "
                         "mean field's bz maps")
    grid = tuple(int(v) for v in np.asarray(kp_grid).reshape(-1))
    if int(np.prod(grid)) != nk:
        raise ValueError("kp_grid does not match the number of k-points of the file")
    kpts = np.asarray(d["kpts"], np.float64).reshape(nk, 3) if "kpts" in d else None
    if kpts is None:
        raise ValueError("thc_reader_t::read(): missing kpts")
    chi_bar = (h5lite.as_complex(d["dual_interpolating_vectors_G0"]).reshape(-1, Np)
               if "dual_interpolating_vectors_G0" in d else None)
    chi_head = (h5lite.as_complex(d["interpolating_vectors_G0"]).reshape(-1, Np)[0]
                if "interpolating_vectors_G0" in d else None)
    if bz is not None:
        if int(bz["nk_ibz"]) != nk_ibz or int(bz["nq_ibz"]) != nq_ibz or \
                V.shape[0] != nq_ibz or len(bz["lex"]) != nk:
            raise ValueError("the bz maps do not match the file's nkpts, nkpts_ibz, nqpts_ibz")
        lex = np.asarray(bz["lex"], np.int64)
        rep = np.asarray(bz["qp_to_ibz"], np.int64)  # 1st-BZ q -> its IBZ point

        def to_lex(a):  # leading axis in the mean field's order -> lexicographic order
            out = np.empty_like(a)
            out[lex] = a
            return out
        X = np.ascontiguousarray(np.swapaxes(to_lex(np.swapaxes(X, 0, 1)), 0, 1))
        V = to_lex(V[rep])
        kpts = to_lex(kpts)
        if chi_bar is not None:
            chi_bar = to_lex(chi_bar[rep] if chi_bar.shape[0] == nq_ibz else chi_bar)
    return THCData(X=np.ascontiguousarray(X), V=np.ascontiguousarray(V), kpts=kpts,
                   lattv=np.asarray(lattv, np.float64), kp_grid=grid, chi_bar=chi_bar,
                   madelung=float(madelung), chi_head=chi_head, bz=bz,
                   bz_rotations=bz_rotations)
