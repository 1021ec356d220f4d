"""ctypes binding of the C ABI declared in include/coqui_b200.h.

Loading fails loudly (ImportError) when the in-tree library has not been built: there is
no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libcoqui_b200.so")

OK = 0
ERRORS = {
    -1: "EINVAL", -2: "EUNSUPPORTED", -3: "ECUDA", -4: "ENOMEM", -5: "ENOTHPD", -6: "EPHSYM",
    -7: "ETIMEDOUT",
}
FP64, MIXED = 0, 1

# Every exported entry point of include/coqui_b200.h.
SYMBOLS = [
    "coqui_b200_create", "coqui_b200_destroy", "coqui_b200_last_error", "coqui_b200_version",
    "coqui_b200_set_ir", "coqui_b200_set_kmesh", "coqui_b200_set_thc", "coqui_b200_eval_pi",
    "coqui_b200_update_w", "coqui_b200_eval_sigma", "coqui_b200_set_w", "coqui_b200_rpa_energy",
    "coqui_b200_primary_to_aux", "coqui_b200_aux_to_primary", "coqui_b200_tau_to_w",
    "coqui_b200_w_to_tau", "coqui_b200_dyson_w", "coqui_b200_last_timings",
    "coqui_b200_kernel_launches", "coqui_b200_gw_iteration", "coqui_b200_set_profiling",
    "coqui_b200_kernel_stats", "coqui_b200_kernel_units", "coqui_b200_set_gcache_limit",
    "coqui_b200_primary_to_aux_noalloc",
    "coqui_b200_set_ir_fermi", "coqui_b200_set_mean_field", "coqui_b200_set_iter_alg",
    "coqui_b200_hf_evaluate", "coqui_b200_scgw_set_hf", "coqui_b200_set_div_treatment",
    "coqui_b200_scgw_iteration", "coqui_b200_get_scgw_state", "coqui_b200_dyson_g",
    "coqui_b200_gm_energy", "coqui_b200_mlp_create", "coqui_b200_mlp_destroy",
    "coqui_b200_mlp_last_error", "coqui_b200_mlp_num_params", "coqui_b200_mlp_set_params",
    "coqui_b200_mlp_get_params", "coqui_b200_mlp_forward", "coqui_b200_mlp_gradient",
    "coqui_b200_mlp_train", "coqui_b200_mlp_extrapolate", "coqui_b200_scgw_set_mlp",
    "coqui_b200_scgw_sigma_diag_w", "coqui_b200_batch_create", "coqui_b200_batch_destroy",
    "coqui_b200_batch_last_error", "coqui_b200_batch_set_ir", "coqui_b200_batch_set_thc",
    "coqui_b200_batch_gw_iteration", "coqui_b200_batch_last_ms", "coqui_b200_set_autotune",
    "coqui_b200_tuned_shapes", "coqui_b200_set_tile_config", "coqui_b200_num_tile_configs",
    "coqui_b200_set_wait_limit_ns", "coqui_b200_factor_dielectric", "coqui_b200_qp_solve",
    "coqui_b200_set_symmetry",
]


class Dims(ctypes.Structure):
    _fields_ = [("ns", ctypes.c_int64), ("nk", ctypes.c_int64), ("nb", ctypes.c_int64),
                ("Np", ctypes.c_int64), ("nt_f", ctypes.c_int64), ("nw_b", ctypes.c_int64),
                ("kp_grid", ctypes.c_int64 * 3), ("precision_mode", ctypes.c_int32),
                ("device", ctypes.c_int32)]


class Symmetry(ctypes.Structure):
    """coqui_b200_symmetry: the mean field's bz_symm maps in the reference's k order."""
    _fields_ = [("nk_ibz", ctypes.c_int64), ("nq_ibz", ctypes.c_int64), ("nsym", ctypes.c_int64),
                ("ld_Qs", ctypes.c_int64), ("k_lex", ctypes.c_void_p),
                ("kp_to_ibz", ctypes.c_void_p), ("kp_trev", ctypes.c_void_p),
                ("kp_trev_pair", ctypes.c_void_p), ("qp_to_ibz", ctypes.c_void_p),
                ("qp_trev", ctypes.c_void_p), ("qminus", ctypes.c_void_p),
                ("nq_per_s", ctypes.c_void_p), ("Qs", ctypes.c_void_p),
                ("ks_to_k", ctypes.c_void_p), ("D", ctypes.c_void_p)]


class CoquiB200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m coqui_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    lib.coqui_b200_create.argtypes = [ctypes.POINTER(P), ctypes.POINTER(Dims)]
    lib.coqui_b200_destroy.argtypes = [P]
    lib.coqui_b200_destroy.restype = None
    lib.coqui_b200_last_error.argtypes = [P]
    lib.coqui_b200_last_error.restype = ctypes.c_char_p
    lib.coqui_b200_version.restype = ctypes.c_char_p
    lib.coqui_b200_set_ir.argtypes = [P, P, P, P, P]
    lib.coqui_b200_set_kmesh.argtypes = [P, P, P, P]
    lib.coqui_b200_set_thc.argtypes = [P, P, P]
    lib.coqui_b200_eval_pi.argtypes = [P, P, P]
    lib.coqui_b200_update_w.argtypes = [P, P, P, P]
    lib.coqui_b200_eval_sigma.argtypes = [P, P, P]
    lib.coqui_b200_set_w.argtypes = [P, P]
    lib.coqui_b200_rpa_energy.argtypes = [P, P, ctypes.POINTER(ctypes.c_double)]
    lib.coqui_b200_primary_to_aux.argtypes = [P, ctypes.c_int64, P, P]
    lib.coqui_b200_aux_to_primary.argtypes = [P, ctypes.c_int64, P, P]
    lib.coqui_b200_tau_to_w.argtypes = [P, P, P]
    lib.coqui_b200_w_to_tau.argtypes = [P, P, P]
    lib.coqui_b200_dyson_w.argtypes = [P, P, P]
    lib.coqui_b200_last_timings.argtypes = [P, ctypes.c_char_p, ctypes.c_int, P, ctypes.c_int]
    lib.coqui_b200_gw_iteration.argtypes = [P, P, P, P]
    lib.coqui_b200_set_profiling.argtypes = [P, ctypes.c_int]
    lib.coqui_b200_kernel_stats.argtypes = [P, ctypes.c_char_p, ctypes.c_int, P, P, ctypes.c_int]
    lib.coqui_b200_kernel_units.argtypes = [P, ctypes.c_char_p, ctypes.c_int, P, ctypes.c_int]
    lib.coqui_b200_set_gcache_limit.argtypes = [P, ctypes.c_int64]
    lib.coqui_b200_primary_to_aux_noalloc.argtypes = [P, P, P, ctypes.c_int64, ctypes.c_int64,
                                                      ctypes.c_int64, P, ctypes.c_char_p,
                                                      ctypes.c_int]
    D, I64 = ctypes.c_double, ctypes.c_int64
    lib.coqui_b200_set_ir_fermi.argtypes = [P, P, P, P, I64, D]
    lib.coqui_b200_set_mean_field.argtypes = [P, P, P, P, D]
    lib.coqui_b200_set_iter_alg.argtypes = [P, ctypes.c_int, D, I64, I64]
    lib.coqui_b200_hf_evaluate.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, D, P]
    lib.coqui_b200_scgw_set_hf.argtypes = [P, ctypes.c_int, ctypes.c_int, D]
    lib.coqui_b200_set_div_treatment.argtypes = [P, ctypes.c_int, D, P]
    lib.coqui_b200_scgw_iteration.argtypes = [P, P, I64, P]
    lib.coqui_b200_get_scgw_state.argtypes = [P, P, P, P]
    lib.coqui_b200_dyson_g.argtypes = [P, P, P, P]
    lib.coqui_b200_gm_energy.argtypes = [P, P, P, ctypes.POINTER(D)]
    lib.coqui_b200_mlp_create.argtypes = [ctypes.POINTER(P), I64, I64, I64, ctypes.c_uint64,
                                          ctypes.c_int]
    lib.coqui_b200_mlp_destroy.argtypes = [P]
    lib.coqui_b200_mlp_destroy.restype = None
    lib.coqui_b200_mlp_last_error.argtypes = [P]
    lib.coqui_b200_mlp_last_error.restype = ctypes.c_char_p
    lib.coqui_b200_mlp_num_params.argtypes = [P]
    lib.coqui_b200_mlp_num_params.restype = I64
    lib.coqui_b200_mlp_set_params.argtypes = [P, P]
    lib.coqui_b200_mlp_get_params.argtypes = [P, P]
    lib.coqui_b200_mlp_forward.argtypes = [P, P, I64, P]
    lib.coqui_b200_mlp_gradient.argtypes = [P, P, P, I64, ctypes.POINTER(ctypes.c_float), P]
    lib.coqui_b200_mlp_train.argtypes = [P, P, P, I64, I64, I64, D, ctypes.c_uint64, P]
    lib.coqui_b200_mlp_extrapolate.argtypes = [P, P, I64, D, P]
    lib.coqui_b200_scgw_set_mlp.argtypes = [P, P, ctypes.c_int, D]
    lib.coqui_b200_scgw_sigma_diag_w.argtypes = [P, P]
    lib.coqui_b200_batch_create.argtypes = [ctypes.POINTER(P), I64, P, P, I64, I64, ctypes.c_int]
    lib.coqui_b200_batch_destroy.argtypes = [P]
    lib.coqui_b200_batch_destroy.restype = None
    lib.coqui_b200_batch_last_error.argtypes = [P]
    lib.coqui_b200_batch_last_error.restype = ctypes.c_char_p
    lib.coqui_b200_batch_set_ir.argtypes = [P, P, P, P]
    lib.coqui_b200_batch_set_thc.argtypes = [P, I64, P, P]
    lib.coqui_b200_batch_gw_iteration.argtypes = [P, P, P]
    lib.coqui_b200_batch_last_ms.argtypes = [P]
    lib.coqui_b200_batch_last_ms.restype = D
    lib.coqui_b200_set_autotune.argtypes = [ctypes.c_int]
    lib.coqui_b200_set_autotune.restype = None
    lib.coqui_b200_tuned_shapes.argtypes = []
    lib.coqui_b200_tuned_shapes.restype = I64
    lib.coqui_b200_set_tile_config.argtypes = [ctypes.c_int]
    lib.coqui_b200_set_tile_config.restype = ctypes.c_int
    lib.coqui_b200_num_tile_configs.argtypes = []
    lib.coqui_b200_num_tile_configs.restype = ctypes.c_int
    lib.coqui_b200_set_wait_limit_ns.argtypes = [ctypes.c_int, I64]
    lib.coqui_b200_set_wait_limit_ns.restype = ctypes.c_int
    lib.coqui_b200_factor_dielectric.argtypes = [P, P, P, P, P, I64, I64, P]
    lib.coqui_b200_factor_dielectric.restype = ctypes.c_int
    lib.coqui_b200_qp_solve.argtypes = [P, P, P, P, I64, ctypes.c_int, D, D, D, ctypes.c_int,
                                        ctypes.c_int, P, P, P, ctypes.c_char_p, ctypes.c_int]
    lib.coqui_b200_qp_solve.restype = ctypes.c_int
    lib.coqui_b200_kernel_launches.argtypes = [P]
    lib.coqui_b200_kernel_launches.restype = ctypes.c_int64
    lib.coqui_b200_set_symmetry.argtypes = [P, ctypes.POINTER(Symmetry)]
    lib.coqui_b200_set_symmetry.restype = ctypes.c_int
    _lib = lib
    return lib


def _ptr(a, name):
    if a is None:
        return None
    if not isinstance(a, np.ndarray) or not a.flags.c_contiguous:
        raise ValueError(f"{name} must be a C-contiguous numpy array")
    return a.ctypes.data


def _c128(a, shape, name):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if tuple(a.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {a.shape}, expected {tuple(shape)}")
    return a


_DIV = {"ignore_g0": 0, "gygi": 1}
_DIV_ALL = {"ignore_g0": 0, "gygi": 1, "gygi_extrplt": 2, "gygi_extrplt_2d": 3}


class Context:
    """One device context: THC data, IR grid, k-mesh and device buffers of one system."""

    def __init__(self, nk, nb, Np, nt_f, nw_b, kp_grid, mode=MIXED, device=0, ns=1):
        self.lib = load()
        d = Dims(ns=ns, nk=nk, nb=nb, Np=Np, nt_f=nt_f, nw_b=nw_b,
                 kp_grid=(ctypes.c_int64 * 3)(*kp_grid), precision_mode=mode, device=device)
        self.h = ctypes.c_void_p()
        rc = self.lib.coqui_b200_create(ctypes.byref(self.h), ctypes.byref(d))
        if rc != OK:
            raise CoquiB200Error(rc, "coqui_b200_create failed")
        self.nk, self.nb, self.Np, self.nt, self.nw_b = nk, nb, Np, nt_f, nw_b
        self.nt_half, self.nw_half = (nt_f + 1) // 2, (nw_b + 1) // 2
        self.mode = mode
        # k-points of G / Sigma and q-points of Pi / W: the IBZ ones after set_symmetry
        self.nkg = self.nqw = nk

    def close(self):
        if self.h:
            self.lib.coqui_b200_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != OK:
            raise CoquiB200Error(rc, self.lib.coqui_b200_last_error(self.h).decode())

    # -- set-up ------------------------------------------------------------------------
    def set_ir(self, ft):
        nt, nw = self.nt, self.nw_b
        Twt = _c128(ft.Twt_bb, (nw, nt), "Twt_bb")
        Ttw = _c128(ft.Ttw_bb, (nt, nw), "Ttw_bb")
        Tb = _c128(ft.T_beta_t_ff, (nt,), "T_beta_t_ff")
        x = np.ascontiguousarray(ft.tau_mesh_x, np.float64)
        self._check(self.lib.coqui_b200_set_ir(self.h, _ptr(Twt, "Twt"), _ptr(Ttw, "Ttw"),
                                               _ptr(Tb, "Tb"), _ptr(x, "tau")))

    def set_ir_fermi(self, ft):
        """Fermionic IR tables of the self-consistent loop (Twt_ff, Ttw_ff, wn_mesh_f, beta)."""
        nt, nw = self.nt, int(ft.Twt_ff.shape[0])
        Twt = _c128(ft.Twt_ff, (nw, nt), "Twt_ff")
        Ttw = _c128(ft.Ttw_ff, (nt, nw), "Ttw_ff")
        wn = np.ascontiguousarray(ft.wn_mesh_f, np.int64).reshape(nw)
        self.nw_f = nw
        self._check(self.lib.coqui_b200_set_ir_fermi(self.h, _ptr(Twt, "Twt"), _ptr(Ttw, "Ttw"),
                                                     _ptr(wn, "wn"), nw, float(ft.beta)))

    def set_mean_field(self, H0, S, F, mu=0.0):
        sh = (1, self.nk, self.nb, self.nb)
        H0, S, F = _c128(H0, sh, "H0"), _c128(S, sh, "S"), _c128(F, sh, "F")
        self._check(self.lib.coqui_b200_set_mean_field(self.h, _ptr(H0, "H0"), _ptr(S, "S"),
                                                       _ptr(F, "F"), float(mu)))

    def set_iter_alg(self, alg="damping", mixing=0.7, max_subsp=5, diis_start=5):
        a = {"damping": 0, "diis": 1}[alg]
        self._check(self.lib.coqui_b200_set_iter_alg(self.h, a, float(mixing), int(max_subsp),
                                                     int(diis_start)))

    def hf_evaluate(self, Dm, S=None, hartree=True, exchange=True, div="ignore_g0",
                    madelung=0.0):
        """THC Hartree-Fock F = J + K of the density matrix Dm (1, nk, nb, nb); div "gygi"
        adds -madelung S Dm S to the exchange."""
        sh = (1, self.nk, self.nb, self.nb)
        Dm = _c128(Dm, sh, "Dm")
        S = None if S is None else _c128(S, sh, "S")
        F = np.empty(sh, np.complex128)
        self._check(self.lib.coqui_b200_hf_evaluate(
            self.h, _ptr(Dm, "Dm"), _ptr(S, "S"), int(bool(hartree)), int(bool(exchange)),
            _DIV[div], float(madelung), _ptr(F, "F")))
        return F

    def set_div_treatment(self, div="ignore_g0", madelung=0.0, chi_head=None):
        """q -> 0 treatment of the eps^-1 head and of Sigma; chi_head (Np) is basis_head at
        q = 0, needed by the gygi corrections of Sigma."""
        chi = None if chi_head is None else _c128(chi_head, (self.Np,), "chi_head")
        self._check(self.lib.coqui_b200_set_div_treatment(self.h, _DIV_ALL[div], float(madelung),
                                                          _ptr(chi, "chi_head")))

    def set_hf(self, enable=True, div="ignore_g0", madelung=0.0):
        """Re-evaluate F = J + K from the density matrix at the start of every scGW iteration."""
        self._check(self.lib.coqui_b200_scgw_set_hf(self.h, int(bool(enable)), _DIV[div],
                                                    float(madelung)))

    def scgw_iteration(self, it, G=None):
        """One self-consistent GW iteration; G (iteration 1) uploads the starting G."""
        G = None if G is None else self._G(G)
        st = np.zeros(8, np.float64)
        self._check(self.lib.coqui_b200_scgw_iteration(self.h, _ptr(G, "G"), int(it), _ptr(st, "st")))
        return dict(conv_F=st[0], conv_Sigma=st[1], e_1e=st[2], e_hf=st[3], e_corr=st[4],
                    e_tot=st[2] + st[3] + st[4], residual=st[5], learned=int(st[6]),
                    evaluations=int(st[7]))

    def set_mlp(self, mlp, enable=True, max_jump=5.0):
        """Learned update of the damped loop (mlp: capi.Mlp with 4 inputs, 2 outputs)."""
        h = mlp.h if (mlp is not None and enable) else None
        self._check(self.lib.coqui_b200_scgw_set_mlp(self.h, h, 1 if enable else 0, float(max_jump)))
        self._mlp_ref = mlp  # the network must outlive its use

    def sigma_diag_w(self):
        out = np.empty((self.nw_f, self.nk, self.nb), np.complex128)
        self._check(self.lib.coqui_b200_scgw_sigma_diag_w(self.h, _ptr(out, "out")))
        return out

    def get_scgw_state(self):
        G = np.empty((self.nt, 1, self.nk, self.nb, self.nb), np.complex128)
        S = np.empty_like(G)
        Dm = np.empty((1, self.nk, self.nb, self.nb), np.complex128)
        self._check(self.lib.coqui_b200_get_scgw_state(self.h, _ptr(G, "G"), _ptr(S, "S"),
                                                       _ptr(Dm, "Dm")))
        return G, S, Dm

    def dyson_g(self, Sigma):
        S = self._G(Sigma)
        G = np.empty_like(S)
        Dm = np.empty((1, self.nk, self.nb, self.nb), np.complex128)
        self._check(self.lib.coqui_b200_dyson_g(self.h, _ptr(S, "Sigma"), _ptr(G, "G"),
                                                _ptr(Dm, "Dm")))
        return G, Dm

    def gm_energy(self, G, Sigma):
        G, S = self._G(G), self._G(Sigma)
        e = ctypes.c_double(0.0)
        self._check(self.lib.coqui_b200_gm_energy(self.h, _ptr(G, "G"), _ptr(S, "Sigma"),
                                                  ctypes.byref(e)))
        return e.value

    def set_kmesh(self, kpts, lattv, chi_bar=None):
        k = np.ascontiguousarray(kpts, np.float64).reshape(self.nk, 3)
        L = np.ascontiguousarray(lattv, np.float64).reshape(3, 3)
        c = None if chi_bar is None else _c128(chi_bar, (self.nk, self.Np), "chi_bar")
        self._check(self.lib.coqui_b200_set_kmesh(self.h, _ptr(k, "kpts"), _ptr(L, "lattv"),
                                                  _ptr(c, "chi")))

    def set_thc(self, X, V):
        X = _c128(X, (1, self.nk, self.Np, self.nb), "X")
        V = _c128(V, (self.nk, self.Np, self.Np), "V")
        self._check(self.lib.coqui_b200_set_thc(self.h, _ptr(X, "X"), _ptr(V, "V")))

    def set_symmetry(self, sym, D=None):
        """Switch to the IBZ k-space path (coqui_b200_set_symmetry) with the bz_symm maps of
        ``sym`` (keys ``k_lex`` or ``lex``, ``nk_ibz``, ``nq_ibz``, ``kp_to_ibz``, ``kp_trev``,
        ``kp_trev_pair``, ``qp_to_ibz``, ``qp_trev``, ``qminus``, ``nq_per_s``, ``Qs``,
        ``ks_to_k``) and the rotations D (nsym, nk_ibz, nb, nb) or None; sym = None returns
        to the full-BZ path.  G / Sigma then cover the IBZ k-points, Pi / W the IBZ q-points."""
        if sym is None:
            self._check(self.lib.coqui_b200_set_symmetry(self.h, None))
            self.nkg = self.nqw = self.nk
            self._sym_keep = None
            return
        i64 = lambda a: np.ascontiguousarray(a, np.int64)  # noqa: E731
        i32 = lambda a: np.ascontiguousarray(np.asarray(a).astype(np.int32))  # noqa: E731
        keep = dict(k_lex=i64(sym["k_lex"] if "k_lex" in sym else sym["lex"]),
                    kp_to_ibz=i64(sym["kp_to_ibz"]), kp_trev=i32(sym["kp_trev"]),
                    kp_trev_pair=i64(sym["kp_trev_pair"]), qp_to_ibz=i64(sym["qp_to_ibz"]),
                    qp_trev=i32(sym["qp_trev"]), qminus=i64(sym["qminus"]),
                    nq_per_s=i64(sym["nq_per_s"]), Qs=i64(np.atleast_2d(sym["Qs"])),
                    ks_to_k=i64(np.atleast_2d(sym["ks_to_k"])))
        nsym = int(keep["nq_per_s"].shape[0])
        nk_ibz, nq_ibz = int(sym["nk_ibz"]), int(sym["nq_ibz"])
        if D is not None:
            keep["D"] = _c128(D, (nsym, nk_ibz, self.nb, self.nb), "D")
        s = Symmetry(nk_ibz=nk_ibz, nq_ibz=nq_ibz, nsym=nsym, ld_Qs=keep["Qs"].shape[1],
                     D=None if D is None else keep["D"].ctypes.data,
                     **{k: keep[k].ctypes.data for k in keep if k != "D"})
        self._check(self.lib.coqui_b200_set_symmetry(self.h, ctypes.byref(s)))
        self._sym_keep = keep
        self.nkg, self.nqw = nk_ibz, nq_ibz

    # -- solvers -----------------------------------------------------------------------
    def _G(self, G):
        return _c128(G, (self.nt, 1, self.nkg, self.nb, self.nb), "G_tskij")

    def eval_pi(self, G, out=None):
        G = self._G(G)
        if out is None:
            out = np.empty((self.nt_half, self.nqw, self.Np, self.Np), np.complex128)
        self._check(self.lib.coqui_b200_eval_pi(self.h, _ptr(G, "G"), _ptr(out, "Pi")))
        return out

    def update_w(self, G, want_w=True, want_head=True, out=None):
        G = self._G(G)
        W = None
        if want_w:
            W = out if out is not None else np.empty((self.nqw, self.nt_half, self.Np, self.Np),
                                                     np.complex128)
        head = np.empty(self.nt_half, np.complex128) if want_head else None
        self._check(self.lib.coqui_b200_update_w(self.h, _ptr(G, "G"), _ptr(W, "W"),
                                                 _ptr(head, "head")))
        return W, head

    def set_w(self, dW_qtPQ):
        W = _c128(dW_qtPQ, (self.nqw, self.nt_half, self.Np, self.Np), "dW_qtPQ")
        self._check(self.lib.coqui_b200_set_w(self.h, _ptr(W, "W")))

    def eval_sigma(self, G, out=None):
        """G = None reuses the device-resident G of the previous call."""
        G = None if G is None else self._G(G)
        if out is None:
            out = np.empty((self.nt, 1, self.nkg, self.nb, self.nb), np.complex128)
        self._check(self.lib.coqui_b200_eval_sigma(self.h, _ptr(G, "G"), _ptr(out, "Sigma")))
        return out

    def rpa_energy(self, G):
        """G = None reuses the device-resident G of the previous call."""
        G = None if G is None else self._G(G)
        e = ctypes.c_double(0.0)
        self._check(self.lib.coqui_b200_rpa_energy(self.h, _ptr(G, "G"), ctypes.byref(e)))
        return e.value

    def gw_iteration(self, G, sigma_out=None, want_sigma=True, want_head=False):
        """update_w + evaluate.  G = None reuses the device-resident G; with want_sigma False
        Sigma stays on the device.  Returns (Sigma or None, eps_inv_head or None)."""
        G = None if G is None else self._G(G)
        S = None
        if want_sigma:
            S = sigma_out if sigma_out is not None else np.empty(
                (self.nt, 1, self.nkg, self.nb, self.nb), np.complex128)
        head = np.empty(self.nt_half, np.complex128) if want_head else None
        self._check(self.lib.coqui_b200_gw_iteration(self.h, _ptr(G, "G"), _ptr(S, "Sigma"),
                                                     _ptr(head, "head")))
        return S, head

    def set_profiling(self, on: bool):
        self._check(self.lib.coqui_b200_set_profiling(self.h, 1 if on else 0))

    def kernel_stats(self):
        """{name: (total_ms, launch_groups)} accumulated while profiling was on."""
        n, L = 64, 48
        names = ctypes.create_string_buffer(n * L)
        ms = np.zeros(n)
        cnt = np.zeros(n, np.int64)
        k = self.lib.coqui_b200_kernel_stats(self.h, names, L, ms.ctypes.data, cnt.ctypes.data, n)
        raw = names.raw
        return {raw[i * L:(i + 1) * L].split(b"\0")[0].decode(): (float(ms[i]), int(cnt[i]))
                for i in range(k)}

    def set_gcache_limit(self, nbytes: int):
        """Bytes of device memory for the projected-G cache (-1: half the free memory, 0: none)."""
        self._check(self.lib.coqui_b200_set_gcache_limit(self.h, int(nbytes)))

    def kernel_units(self):
        """{name: work units} accumulated while profiling was on: the (tau, k) problems of the
        projection groups (0 for groups that do not count theirs)."""
        n, L = 64, 48
        names = ctypes.create_string_buffer(n * L)
        units = np.zeros(n, np.int64)
        k = self.lib.coqui_b200_kernel_units(self.h, names, L, units.ctypes.data, n)
        raw = names.raw
        return {raw[i * L:(i + 1) * L].split(b"\0")[0].decode(): int(units[i]) for i in range(k)}

    def primary_to_aux(self, O_tskab):
        O = np.ascontiguousarray(O_tskab, np.complex128)
        nt = O.size // (self.nk * self.nb * self.nb)
        O = O.reshape(nt, 1, self.nk, self.nb, self.nb)
        out = np.empty((nt, 1, self.nk, self.Np, self.Np), np.complex128)
        self._check(self.lib.coqui_b200_primary_to_aux(self.h, nt, _ptr(O, "O"), _ptr(out, "out")))
        return out

    def aux_to_primary(self, O_tskPQ):
        O = np.ascontiguousarray(O_tskPQ, np.complex128)
        nt = O.size // (self.nk * self.Np * self.Np)
        O = O.reshape(nt, 1, self.nk, self.Np, self.Np)
        out = np.empty((nt, 1, self.nk, self.nb, self.nb), np.complex128)
        self._check(self.lib.coqui_b200_aux_to_primary(self.h, nt, _ptr(O, "O"), _ptr(out, "out")))
        return out

    def tau_to_w(self, X_tqPQ):
        X = _c128(X_tqPQ, (self.nt_half, self.nk, self.Np, self.Np), "X_tqPQ")
        out = np.empty((self.nw_half, self.nk, self.Np, self.Np), np.complex128)
        self._check(self.lib.coqui_b200_tau_to_w(self.h, _ptr(X, "X"), _ptr(out, "out")))
        return out

    def w_to_tau(self, X_wqPQ):
        X = _c128(X_wqPQ, (self.nw_half, self.nk, self.Np, self.Np), "X_wqPQ")
        out = np.empty((self.nt_half, self.nk, self.Np, self.Np), np.complex128)
        self._check(self.lib.coqui_b200_w_to_tau(self.h, _ptr(X, "X"), _ptr(out, "out")))
        return out

    def dyson_w(self, Pi_wqPQ):
        P = _c128(Pi_wqPQ, (self.nw_half, self.nk, self.Np, self.Np), "Pi_wqPQ")
        out = np.empty_like(P)
        self._check(self.lib.coqui_b200_dyson_w(self.h, _ptr(P, "Pi"), _ptr(out, "W")))
        return out

    # -- introspection -----------------------------------------------------------------
    def timings(self):
        n, L = 32, 48
        names = ctypes.create_string_buffer(n * L)
        ms = np.zeros(n)
        k = self.lib.coqui_b200_last_timings(self.h, names, L, ms.ctypes.data, n)
        raw = names.raw
        return [(raw[i * L:(i + 1) * L].split(b"\0")[0].decode(), float(ms[i])) for i in range(k)]

    def kernel_launches(self) -> int:
        return int(self.lib.coqui_b200_kernel_launches(self.h))


def primary_to_aux_noalloc(X_ptr, G_ptr, out_ptr, nk, Np, nb, stream=None):
    """Projection O = X G X^H on device buffers the caller owns, with no device allocation.

    X_ptr (complex128 (nk, Np, nb)), G_ptr (complex128 (nk, nb, nb)) and out_ptr
    (complex64 (nk, Np, Np)) are device addresses (ints).  For callers that must not
    allocate device memory; intermediates use the library's fixed 32 MiB device array."""
    lib = load()
    err = ctypes.create_string_buffer(256)
    rc = lib.coqui_b200_primary_to_aux_noalloc(X_ptr, G_ptr, out_ptr, nk, Np, nb, stream, err, 256)
    if rc != OK:
        raise CoquiB200Error(rc, err.value.decode())


def version() -> str:
    return load().coqui_b200_version().decode()


class Mlp:
    """The learned self-energy update's network (in -> width -> width -> out, tanh), trained
    and evaluated on the device by the library's own kernels."""

    def __init__(self, din=4, width=256, dout=2, seed=0, device=0):
        self.lib = load()
        self.din, self.width, self.dout = din, width, dout
        self.h = ctypes.c_void_p()
        rc = self.lib.coqui_b200_mlp_create(ctypes.byref(self.h), din, width, dout, seed, device)
        if rc != OK:
            raise CoquiB200Error(rc, "coqui_b200_mlp_create failed")
        self.nparam = int(self.lib.coqui_b200_mlp_num_params(self.h))

    def close(self):
        if self.h:
            self.lib.coqui_b200_mlp_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != OK:
            raise CoquiB200Error(rc, self.lib.coqui_b200_mlp_last_error(self.h).decode())

    def params(self):
        p = np.empty(self.nparam, np.float32)
        self._check(self.lib.coqui_b200_mlp_get_params(self.h, _ptr(p, "params")))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32).reshape(self.nparam)
        self._check(self.lib.coqui_b200_mlp_set_params(self.h, _ptr(p, "params")))

    def forward(self, X):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, self.din)
        Y = np.empty((X.shape[0], self.dout), np.float32)
        self._check(self.lib.coqui_b200_mlp_forward(self.h, _ptr(X, "X"), X.shape[0], _ptr(Y, "Y")))
        return Y

    def gradient(self, X, T):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, self.din)
        T = np.ascontiguousarray(T, np.float32).reshape(-1, self.dout)
        g = np.empty(self.nparam, np.float32)
        loss = ctypes.c_float(0.0)
        self._check(self.lib.coqui_b200_mlp_gradient(self.h, _ptr(X, "X"), _ptr(T, "T"), X.shape[0],
                                                     ctypes.byref(loss), _ptr(g, "g")))
        return loss.value, g

    def extrapolate(self, hist, max_jump=5.0):
        """hist (4, n) complex128, oldest first -> learned correction (n,) complex128."""
        h = np.ascontiguousarray(hist, np.complex128)
        n = h.shape[1]
        out = np.empty(n, np.complex128)
        self._check(self.lib.coqui_b200_mlp_extrapolate(self.h, _ptr(h, "hist"), n,
                                                        float(max_jump), _ptr(out, "delta")))
        return out

    def train(self, X, T, batch=4096, epochs=10, lr=1e-3, seed=0):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, self.din)
        T = np.ascontiguousarray(T, np.float32).reshape(-1, self.dout)
        hist = np.zeros(epochs, np.float32)
        self._check(self.lib.coqui_b200_mlp_train(self.h, _ptr(X, "X"), _ptr(T, "T"), X.shape[0],
                                                  batch, epochs, float(lr), seed, _ptr(hist, "h")))
        return hist


class Batch:
    """Uneven batch of Gamma-only molecules run with fused launches (mixed precision)."""

    def __init__(self, nb, Np, nt_f, nw_b, device=0):
        self.lib = load()
        self.nb = [int(v) for v in nb]
        self.Np = [int(v) for v in Np]
        self.nt, self.nw_b = nt_f, nw_b
        a = np.ascontiguousarray(self.nb, np.int64)
        b = np.ascontiguousarray(self.Np, np.int64)
        self.h = ctypes.c_void_p()
        rc = self.lib.coqui_b200_batch_create(ctypes.byref(self.h), len(self.nb), _ptr(a, "nb"),
                                              _ptr(b, "Np"), nt_f, nw_b, device)
        if rc != OK:
            raise CoquiB200Error(rc, "coqui_b200_batch_create failed")

    def close(self):
        if self.h:
            self.lib.coqui_b200_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != OK:
            raise CoquiB200Error(rc, self.lib.coqui_b200_batch_last_error(self.h).decode())

    def set_ir(self, ft):
        nt, nw = self.nt, self.nw_b
        Twt = _c128(ft.Twt_bb, (nw, nt), "Twt_bb")
        Ttw = _c128(ft.Ttw_bb, (nt, nw), "Ttw_bb")
        x = np.ascontiguousarray(ft.tau_mesh_x, np.float64)
        self._check(self.lib.coqui_b200_batch_set_ir(self.h, _ptr(Twt, "Twt"), _ptr(Ttw, "Ttw"),
                                                     _ptr(x, "tau")))

    def set_thc(self, m, X, V):
        X = _c128(X, (self.Np[m], self.nb[m]), "X")
        V = _c128(V, (self.Np[m], self.Np[m]), "V")
        self._check(self.lib.coqui_b200_batch_set_thc(self.h, int(m), _ptr(X, "X"), _ptr(V, "V")))

    def gw_iteration(self, G_list, sigma_out=None):
        """G_list[m] (nt, nb_m, nb_m) complex128 -> list of Sigma (nt, nb_m, nb_m)."""
        Gs = [_c128(G, (self.nt, n, n), "G") for G, n in zip(G_list, self.nb)]
        Ss = sigma_out if sigma_out is not None else [np.empty_like(G) for G in Gs]
        gp = (ctypes.c_void_p * len(Gs))(*[G.ctypes.data for G in Gs])
        sp = (ctypes.c_void_p * len(Ss))(*[S.ctypes.data for S in Ss])
        self._check(self.lib.coqui_b200_batch_gw_iteration(self.h, gp, sp))
        return Ss

    def last_ms(self):
        """Device time of the last gw_iteration (CUDA events), ms."""
        return float(self.lib.coqui_b200_batch_last_ms(self.h))


def set_autotune(on: bool):
    """Tile-shape autotuner of the tensor-core GEMMs (process-wide)."""
    load().coqui_b200_set_autotune(1 if on else 0)


def tuned_shapes() -> int:
    return int(load().coqui_b200_tuned_shapes())


def set_tile_config(cfg: int):
    """Pins every tensor-core GEMM to tile configuration cfg (-1: autotuner / heuristic)."""
    if load().coqui_b200_set_tile_config(int(cfg)) != OK:
        raise ValueError(f"tile configuration {cfg} outside -1 .. {num_tile_configs() - 1}")


def num_tile_configs() -> int:
    return int(load().coqui_b200_num_tile_configs())


def factor_dielectric(M_ptr, A_ptr, logdet_ptr, trace_ptr, info_ptr, Np, nprob, stream=None):
    """Batched FP64 factorisation I - M = C C^H of the Dyson step on device buffers (pointers as
    integers): M complex64 (nprob, Np, Np), A complex128 workspace, logdet float64 (nprob),
    trace complex128 (nprob), info int32 (nprob)."""
    rc = load().coqui_b200_factor_dielectric(M_ptr, A_ptr, logdet_ptr, trace_ptr, info_ptr,
                                             int(Np), int(nprob), stream)
    if rc != OK:
        raise CoquiB200Error(rc, "factor_dielectric failed")


QP_METHODS = {"sc": 0, "sc_bisection": 0, "sc_newton": 1, "linearized": 2, "spectral": 3}


def qp_solve(w_fit, sigma_fit, vhf, e0, mu, eta=1e-4, tol=1e-8, qp_type="sc", device=0):
    """Quasiparticle energies E (nel,) from Sigma(i w_n) at the Pade fit points: w_fit (nfit,)
    real, sigma_fit (nfit, nel) complex, vhf and e0 (nel,) real.  Returns (E, residual,
    converged)."""
    w = np.ascontiguousarray(w_fit, np.float64)
    sig = np.ascontiguousarray(sigma_fit, np.complex128)
    v = np.ascontiguousarray(vhf, np.float64)
    e = np.ascontiguousarray(e0, np.float64)
    nfit, nel = sig.shape
    if w.shape != (nfit,) or v.shape != (nel,) or e.shape != (nel,):
        raise ValueError("qp_solve: inconsistent shapes")
    E = np.empty(nel, np.float64)
    R = np.empty(nel, np.float64)
    C = np.empty(nel, np.int32)
    err = ctypes.create_string_buffer(512)
    rc = load().coqui_b200_qp_solve(_ptr(w, "w"), _ptr(sig, "sigma"), _ptr(v, "vhf"),
                                    _ptr(e, "e0"), nel, nfit, float(mu), float(eta), float(tol),
                                    QP_METHODS[qp_type], int(device), _ptr(E, "E"), _ptr(R, "R"),
                                    _ptr(C, "conv"), err, 512)
    if rc != OK:
        raise CoquiB200Error(rc, err.value.decode())
    return E, R, C.astype(bool)


def set_wait_limit_ns(ns: int, device: int = 0):
    """Time limit of the tensor-core kernels' bounded device waits (ns; <= 0: the default 2 s)."""
    rc = load().coqui_b200_set_wait_limit_ns(int(device), int(ns))
    if rc != OK:
        raise CoquiB200Error(rc, "set_wait_limit_ns failed")
