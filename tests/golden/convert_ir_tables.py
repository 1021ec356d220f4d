"""Convert CoQui's shipped IR sparse-sampling tables (HDF5) into compact .npz files.

The reference reads ``src/numerics/imag_axes_ft/ir/data/{lambda}.{eps}.h5`` at run time
(``src/numerics/imag_axes_ft/ir/ir_driver.hpp:41-66``).  This package ships the same
numbers as ``coqui_b200/ir_data/{lambda}.{eps}.npz`` (written by this script) so that no HDF5 library is needed
where the GPU path runs.  The tables are copied value for value (dimensionless, before
the beta rescaling that ``IAFT`` applies, ``ir_driver.hpp:68-73``).

Usage::

    python tests/golden/convert_ir_tables.py <reference-ir-data-dir> [names...]

``names`` default to the grids the benchmark and test workloads use.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..")
sys.path.insert(0, ROOT)
from coqui_b200.h5lite import as_complex, read_h5  # noqa: E402

DEFAULT_NAMES = ["1e4.1e-06", "1e4.1e-10", "1e4.1e-15", "1e5.1e-06", "1e5.1e-15", "1e3.1e-06"]


def convert(src_dir: str, name: str, out_dir: str) -> str:
    d = read_h5(os.path.join(src_dir, name + ".h5"))
    f, b = d["fermion"], d["boson"]
    out = dict(
        nt_f=np.int64(f["nt"]), nw_f=np.int64(f["nw"]),
        nt_b_file=np.int64(b["nt"]), nw_b=np.int64(b["nw"]),
        tau_mesh_f=np.asarray(f["tau_mesh"], np.float64),
        tau_mesh_b=np.asarray(b["tau_mesh"], np.float64),
        wn_mesh_f=np.asarray(f["wn_mesh"], np.int64),
        wn_mesh_b=np.asarray(b["wn_mesh"], np.int64),
        Ttw_ff=as_complex(f["Ttw"]), Twt_ff=as_complex(f["Twt"]),
        Ttw_bb=as_complex(b["Ttw"]), Twt_bb=as_complex(b["Twt"]),
        T_beta_t_ff=as_complex(f["T_betat"]),
        T_zero_t_ff=np.asarray(f["T_zerot"], np.float64).astype(np.complex128),
        # the reference loads the boson "Tct" from the fermion group (ir_driver.hpp:65)
        Tct_ff=as_complex(f["Tct"]),
    )
    path = os.path.join(out_dir, name + ".npz")
    np.savez_compressed(path, **out)
    return path


def main(argv):
    if len(argv) < 2:
        print(__doc__)
        return 2
    src = argv[1]
    names = argv[2:] or DEFAULT_NAMES
    out_dir = os.path.join(ROOT, "coqui_b200", "ir_data")
    for n in names:
        print(convert(src, n, out_dir))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
