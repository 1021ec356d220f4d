"""Regenerate the golden fixtures under tests/golden/ from the CoQui reference checkout.

Sources (all read-only, in the reference tree):

* ``tests/unit_test_files/pyscf/si_kp222_krhf/gw_Gw_Gt_beta1000_wmax1.2_{high,medium}.h5``
  -- G(tau), G(iw_n) and Dm = -G(beta^-) of a Si 2x2x2 GW run, used by the reference's
  ``src/numerics/imag_axes_ft/tests/test_iaft.cpp:46-119`` (tolerances 1e-11 / 1e-9).
* ``tests/unit_test_files/pyscf/si_kp222_krhf/hf_Gw_Gt_beta1000_wmax1.2_high.h5``
  -- the HF G0(tau) and Dm used by ``src/methods/SCF/tests/test_scf_common.cpp:61-96``
  (tolerance 1e-8).

To keep the fixtures small only k-points {0, 3} are kept (all tau / iw_n points and
full orbital blocks, so every tau<->iw_n transform and the G0 eigen-structure are intact).

Usage::

    python tests/golden/make_golden.py <reference-root>
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from coqui_b200.h5lite import as_complex, read_h5  # noqa: E402

KEEP_K = [0, 3]


def main(argv):
    if len(argv) < 2:
        print(__doc__)
        return 2
    base = os.path.join(argv[1], "tests", "unit_test_files", "pyscf", "si_kp222_krhf")
    for kind, prec in [("gw", "high"), ("gw", "medium"), ("hf", "high")]:
        d = read_h5(os.path.join(base, f"{kind}_Gw_Gt_beta1000_wmax1.2_{prec}.h5"))
        Gt = as_complex(d["Gt"])[:, :, KEEP_K]
        Gw = as_complex(d["Gw"])[:, :, KEEP_K]
        Dm = as_complex(d["Dm"])[:, KEEP_K]
        out = os.path.join(HERE, f"si_kp222_{kind}_G_beta1000_wmax1.2_{prec}.npz")
        np.savez_compressed(out, Gt=Gt, Gw=Gw, Dm=Dm, k_index=np.array(KEEP_K),
                            beta=1000.0, wmax=1.2, prec=prec)
        print(out, Gt.shape, Gw.shape, Dm.shape)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
