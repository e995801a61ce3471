"""Extract the input tables this package ships from a checkout of the reference.

The solver reads only a few keys of the reference's ``data/inputs/final_export.npz``
(``pf_kks/materials.py:33-55``) and only the precipitate centres and radii of
``data/inputs/micro_final.npz`` (``pf_kks/microstructure.py:77-94``). This
script copies exactly those keys, unchanged, into ``final_export.npz`` and
``micro_final.npz`` next to it, so that runs do not need the reference tree.

Usage: python make_data.py /path/to/reference/checkout
"""

import os
import sys

import numpy as np

TABLE_KEYS = ("T", "A_fcc", "B_fcc", "C_fcc", "A_dia", "B_dia", "C_dia", "C11", "C12", "C44", "delta", "Vm", "gamma",
              "X_Si_fcc", "D0", "QD")
MICRO_KEYS = ("ox_cyl", "oy_cyl", "oz_cyl", "r_cyl")


def main(ref_root):
    here = os.path.dirname(os.path.abspath(__file__))
    d = np.load(os.path.join(ref_root, "data", "inputs", "final_export.npz"))
    np.savez(os.path.join(here, "final_export.npz"), **{k: d[k] for k in TABLE_KEYS})
    m = np.load(os.path.join(ref_root, "data", "inputs", "micro_final.npz"))
    np.savez(os.path.join(here, "micro_final.npz"), **{k: m[k] for k in MICRO_KEYS})


if __name__ == "__main__":
    _ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PF_KKS_REFERENCE")
    if not _ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_CHECKOUT (or set PF_KKS_REFERENCE)")
    main(_ref)
