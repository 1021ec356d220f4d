"""Host-side IR imaginary-axis grid (mirror of CoQui's ``imag_axes_ft::IAFT``).

Loads the shipped IR sparse-sampling tables (``ir_data/*.npz``, converted value for value
from the reference's ``src/numerics/imag_axes_ft/ir/data/*.h5``), applies the beta
rescaling of ``ir_driver.hpp:68-73`` and builds the particle-hole symmetric transform
matrices of ``IAFT.icc:61-70`` and ``:116-125`` that the device transforms consume.
Small host-side matrix work only: the tau <-> iw transforms of large tensors run on the GPU.
"""
from __future__ import annotations

import os

import numpy as np

IR_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ir_data")
PREC_FILE = {"high": "1e-15", "medium": "1e-10", "low": "1e-06"}
_LAMBDAS = [(1e2, "1e2"), (1e3, "1e3"), (1e4, "1e4"), (1e5, "1e5"), (1e6, "1e6")]


class IAFT:
    def __init__(self, beta: float, wmax: float, prec: str = "high"):
        if prec not in PREC_FILE:
            raise ValueError(f"prec = {prec} is not acceptable: high, medium, low")
        lam_in = beta * wmax
        for lam, tag in _LAMBDAS:
            if lam_in <= lam:
                break
        else:
            raise ValueError(f"beta*wmax = {lam_in} above 1e6")
        self.beta, self.lam, self.prec = float(beta), lam, prec
        self.wmax = lam / beta
        path = os.path.join(IR_DIR, f"{tag}.{PREC_FILE[prec]}.npz")
        if not os.path.exists(path):
            raise FileNotFoundError(f"IR table {path} not shipped; convert it with tests/golden/convert_ir_tables.py")
        d = np.load(path)
        self.nt_f, self.nw_f, self.nw_b = int(d["nt_f"]), int(d["nw_f"]), int(d["nw_b"])
        self.tau_mesh_x = d["tau_mesh_f"]
        self.wn_mesh_f, self.wn_mesh_b = d["wn_mesh_f"], d["wn_mesh_b"]
        b = self.beta
        self.Ttw_ff = d["Ttw_ff"] * (np.sqrt(2.0) / b)
        self.Twt_ff = d["Twt_ff"] * (b / np.sqrt(2.0))
        self.Ttw_bb = d["Ttw_bb"] * (np.sqrt(2.0) / b)
        self.Twt_bb = d["Twt_bb"] * (b / np.sqrt(2.0))
        self.T_beta_t_ff = d["T_beta_t_ff"]

    # the reference's nt_b() returns nt_f (IAFT.hpp:167-169); the tau meshes coincide
    @property
    def nt_b(self):
        return self.nt_f

    @property
    def nt_half(self):
        return (self.nt_b + 1) // 2

    @property
    def nw_half(self):
        return (self.nw_b + 1) // 2

    def tau_mesh(self):
        return (self.tau_mesh_x + 1.0) * self.beta / 2.0

    def check_ph_symmetric(self):
        """thc_gw.cpp:56-66: |tau_i| == |tau_{n-1-i}| in the [-1, 1] mesh."""
        x = self.tau_mesh_x
        return bool(np.all(np.abs(x) - np.abs(x[::-1]) <= 1e-6))

    def Twt_pos(self):
        nw, nt = self.nw_half, self.nt_half
        n = np.arange(nw)[:, None] + self.nw_b // 2
        it = np.arange(nt)[None, :]
        imt = self.nt_b - it - 1
        T = self.Twt_bb[n, it] + np.where(it == imt, 0.0, self.Twt_bb[n, imt])
        return np.ascontiguousarray(T)

    def Ttw_pos(self):
        nt, nw = self.nt_half, self.nw_half
        it = np.arange(nt)[:, None]
        n = np.arange(nw)[None, :]
        iw, imw = self.nw_b // 2 + n, self.nw_b // 2 - n
        T = self.Ttw_bb[it, iw] + np.where(iw == imw, 0.0, self.Ttw_bb[it, imw])
        return np.ascontiguousarray(T)
