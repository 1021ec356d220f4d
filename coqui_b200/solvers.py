"""Host-side mirror of CoQui's THC-RPA/GW solver interface, backed by the CUDA library.

Names, argument meaning and error behaviour follow the reference (paths relative to the
CoQui tree):

* :class:`THCData` plays ``thc_reader_t`` + ``mf::MF`` (``X``, ``Z``/V, ``basis_bar_head``,
  ``kpts``, ``lattv``, ``kp_grid``; ``src/methods/ERI/thc_reader_t.hpp:590-815``).
* :class:`MBState` holds ``sG_tskij``, ``sSigma_tskij``, ``dW_qtPQ``, ``eps_inv_head``
  (``src/methods/mb_state/mb_state.hpp:79-84``).
* :class:`scr_coulomb_t` has ``update_w``, ``eval_Pi_qdep``, ``tau_to_w``, ``w_to_tau``,
  ``dyson_W_in_place`` (``src/methods/scr_coulomb/scr_coulomb_t.h``).
* :class:`gw_t` has ``evaluate`` and ``rpa_energy`` (``src/methods/GW/gw_t.h:55-75``).
* :class:`hf_t` has the THC ``evaluate`` (``src/methods/HF/hf_t.h:52-56``).

Every call runs on the GPU through :mod:`coqui_b200.capi`; the reference's fatal
``utils::check`` failures surface as :class:`coqui_b200.capi.CoquiB200Error`.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import capi
from .iaft import IAFT

DIV_TREATMENTS = ("ignore_g0", "gygi", "gygi_extrplt", "gygi_extrplt_2d")


@dataclass
class THCData:
    X: np.ndarray  # (ns, nk, Np, nb) complex128 collocation
    V: np.ndarray  # (nq, Np, Np) complex128 Coulomb matrix ("Z" in the reference)
    kpts: np.ndarray  # (nk, 3) cartesian
    lattv: np.ndarray  # (3, 3) rows = lattice vectors
    kp_grid: tuple
    chi_bar: Optional[np.ndarray] = None  # (nq, Np) basis_bar_head
    madelung: float = 0.0  # MF::madelung(), used by the gygi corrections
    chi_head: Optional[np.ndarray] = None  # (Np) basis_head at q = 0 (gygi Sigma correction)
    # MF::bz() maps of a symmetric mean field (keys as coqui_b200.symmetry.bz_symmetry, with
    # "lex" the lexicographic position of each of the mean field's k-points) and the rotations
    # symmetry_rotation(isym, k) as (nsym, nk_ibz, nb, nb); with them update_w / evaluate /
    # rpa_energy take the reference's k-space routes (G, Sigma on the IBZ k-points, W on the
    # IBZ q-points).  X, V, kpts and chi_bar stay on the whole lexicographic grid.
    bz: Optional[dict] = None
    bz_rotations: Optional[np.ndarray] = None

    @property
    def Np(self):
        return self.X.shape[2]

    @property
    def nbnd(self):
        return self.X.shape[3]

    @property
    def nkpts(self):
        return self.X.shape[1]

    @classmethod
    def from_synthetic(cls, s):
        return cls(X=s.X, V=s.V, kpts=s.kpts, lattv=s.lattv, kp_grid=s.kp_grid, chi_bar=s.chi_bar)


@dataclass
class MBState:
    sG_tskij: Optional[np.ndarray] = None
    sSigma_tskij: Optional[np.ndarray] = None
    dW_qtPQ: Optional[np.ndarray] = None
    eps_inv_head: Optional[np.ndarray] = None
    screen_type: str = ""
    meta: dict = field(default_factory=dict)


_ctx_cache: dict = {}


def context_for(thc: THCData, ft: IAFT, mode: int = capi.MIXED, device: int = 0) -> capi.Context:
    """Device context holding thc and ft (created once per (thc, ft, mode, device))."""
    key = (id(thc), id(ft), mode, device)
    ctx = _ctx_cache.get(key)
    if ctx is None:
        ctx = capi.Context(thc.nkpts, thc.nbnd, thc.Np, ft.nt_f, ft.nw_b, thc.kp_grid, mode=mode,
                           device=device)
        ctx.set_ir(ft)
        ctx.set_kmesh(thc.kpts, thc.lattv, thc.chi_bar)
        ctx.set_thc(thc.X, thc.V)
        if thc.bz is not None:  # nqpts_ibz < nqpts: the k-space routes (thc_gw.icc:31-32)
            ctx.set_symmetry(thc.bz, thc.bz_rotations)
        _ctx_cache[key] = ctx
    return ctx


def hf_context_for(thc: THCData, mode: int = capi.MIXED, device: int = 0) -> capi.Context:
    """A context holding thc: any context of the same (thc, mode, device), else one without
    imaginary-time grids (Hartree-Fock needs none)."""
    if thc.bz is not None:
        raise capi.CoquiB200Error(-2, "THC Hartree-Fock takes the whole k-mesh; the "
                                      "symmetry-reduced form is not on this path")
    for (t, _, m, d), ctx in _ctx_cache.items():
        if t == id(thc) and m == mode and d == device:
            return ctx
    key = (id(thc), None, mode, device)
    ctx = capi.Context(thc.nkpts, thc.nbnd, thc.Np, 2, 1, thc.kp_grid, mode=mode, device=device)
    ctx.set_kmesh(thc.kpts, thc.lattv, thc.chi_bar)
    ctx.set_thc(thc.X, thc.V)
    _ctx_cache[key] = ctx
    return ctx


def clear_contexts():
    for c in _ctx_cache.values():
        c.close()
    _ctx_cache.clear()


class scr_coulomb_t:
    """Screened interaction in the THC basis (scr_coulomb_t.cpp)."""

    def __init__(self, ft: IAFT, screen_type: str = "rpa", div_treatment: str = "ignore_g0",
                 mode: int = capi.MIXED):
        if screen_type != "rpa":
            raise ValueError(f"screen_type = {screen_type}: only 'rpa' is on this path")
        if div_treatment not in DIV_TREATMENTS:
            raise ValueError(f"unknown div_treatment {div_treatment}")
        self.ft, self.screen_type, self.div_treatment, self.mode = ft, screen_type, div_treatment, mode

    def update_w(self, mb_state: MBState, thc: THCData, h5_iter: int = -1):
        """scr_coulomb_t.cpp:37-95: fills mb_state.dW_qtPQ and mb_state.eps_inv_head."""
        if mb_state.sG_tskij is None:
            raise capi.CoquiB200Error(-1, "update_w: sG_tskij is not initialized in MBState")
        ctx = context_for(thc, self.ft, self.mode)
        ctx.set_div_treatment(self.div_treatment, thc.madelung, thc.chi_head)
        W, head = ctx.update_w(mb_state.sG_tskij)
        mb_state.dW_qtPQ = W
        mb_state.eps_inv_head = head
        mb_state.screen_type = self.screen_type
        mb_state.meta["w_on_device"] = ctx

    def eval_Pi_qdep(self, G_tskij, thc: THCData):
        return context_for(thc, self.ft, self.mode).eval_pi(G_tskij)

    def tau_to_w(self, Pi_tqPQ, thc: THCData):
        return context_for(thc, self.ft, self.mode).tau_to_w(Pi_tqPQ)

    def w_to_tau(self, W_wqPQ, thc: THCData):
        return context_for(thc, self.ft, self.mode).w_to_tau(W_wqPQ)

    def dyson_W_in_place(self, Pi_wqPQ, thc: THCData):
        return context_for(thc, self.ft, self.mode).dyson_w(Pi_wqPQ)


class gw_t:
    """THC-GW self-energy and THC-RPA energy (thc_gw.cpp, thc_rpa.cpp)."""

    def __init__(self, ft: IAFT, div_treatment: str = "ignore_g0", mode: int = capi.MIXED):
        if div_treatment not in DIV_TREATMENTS:
            raise ValueError(f"unknown div_treatment {div_treatment}")
        self.ft, self.div_treatment, self.mode = ft, div_treatment, mode

    def evaluate(self, mb_state: MBState, thc: THCData, verbose: bool = False):
        """thc_gw.cpp:26-89: overwrites mb_state.sSigma_tskij from sG_tskij and dW_qtPQ."""
        for name in ("sG_tskij", "dW_qtPQ"):
            if getattr(mb_state, name) is None:
                raise capi.CoquiB200Error(-1, f"gw_t::evaluate: {name} is not initialized in MBState")
        if not self.ft.check_ph_symmetric():
            raise capi.CoquiB200Error(-6, "thc-gw: IAFT grid is not compatible with PH symmetry")
        ctx = context_for(thc, self.ft, self.mode)
        ctx.set_div_treatment(self.div_treatment, thc.madelung, thc.chi_head)
        if mb_state.meta.get("w_on_device") is not ctx:
            ctx.set_w(mb_state.dW_qtPQ)
        mb_state.sSigma_tskij = ctx.eval_sigma(mb_state.sG_tskij)

    def rpa_energy(self, G_tskij, thc: THCData) -> float:
        """thc_rpa.cpp:22 / thc_rpa.icc:21-181."""
        return context_for(thc, self.ft, self.mode).rpa_energy(G_tskij)


class hf_t:
    """THC Hartree-Fock (hf_t.h:40-60; thc_hf.cpp:21-60 -> thc_hf.icc:17-272 for q-independent
    THC without symmetry; HF_K_correction hf_t.cpp:45-84).

    As the reference constructor (hf_t.cpp:31-37), a treatment other than "ignore_g0" or
    "gygi" becomes "gygi"."""

    def __init__(self, div_treatment: str = "gygi", mode: int = capi.MIXED):
        if div_treatment not in DIV_TREATMENTS:
            raise ValueError(f"unknown div_treatment {div_treatment}")
        self.div_treatment = div_treatment if div_treatment in ("ignore_g0", "gygi") else "gygi"
        self.mode = mode

    def evaluate(self, sF_skij, Dm_skij, thc: THCData, S_skij, hartree: bool = True,
                 exchange: bool = True):
        """Overwrites sF_skij (ns, nk, nb, nb) with J + K of the density matrix Dm_skij; the
        gygi treatment adds -madelung S Dm S (thc.madelung) to the exchange."""
        ctx = hf_context_for(thc, self.mode)
        F = ctx.hf_evaluate(Dm_skij, S_skij, hartree, exchange, self.div_treatment,
                            thc.madelung)
        sF_skij[...] = F.reshape(np.shape(sF_skij))
        return sF_skij
