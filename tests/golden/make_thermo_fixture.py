"""Generate ``reference_thermo.npz`` from the reference's CALPHAD description:
the functions its simulated DSC evaluates (pf_kks/postprocess/dsc.py:111-119)
on a grid of temperatures and matrix Si fractions.

    python tests/golden/make_thermo_fixture.py REF

REF is a checkout of the reference (or set $PF_KKS_REFERENCE); it is read,
never written. Contents: ``T`` (n), ``x`` (m); ``Hm_fcc``, ``d_Hm_fcc_dSi``,
``cp_fcc``, ``Vmfcc`` (n, m) at (T, x); ``Hm_dia``, ``cp_dia``, ``Vmdia`` (n)
at x = 0.9999, all from ``pf_kks.thermo.gibbs_energy`` / ``molar_volume``
(T0 = 298 K for the volumes, as the DSC uses).
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TEMPERATURES = np.array([300.0, 350.0, 400.0, 450.0, 500.0, 510.0, 520.0, 560.0, 600.0, 650.0, 699.5, 700.0,
                         700.5, 719.0, 760.0, 850.0, 933.0])
FRACTIONS = np.array([1e-5, 1e-4, 1e-3, 0.003, 0.01, 0.02, 0.025, 0.05, 0.1, 0.3])


def main(ref_root):
    sys.path.insert(0, ref_root)
    from pf_kks.thermo import gibbs_energy, molar_volume

    n, m = TEMPERATURES.size, FRACTIONS.size
    out = {"T": TEMPERATURES, "x": FRACTIONS}
    for key in ("Hm_fcc", "d_Hm_fcc_dSi", "cp_fcc", "Vmfcc"):
        out[key] = np.zeros((n, m))
    for key in ("Hm_dia", "cp_dia", "Vmdia"):
        out[key] = np.zeros(n)
    for i, T in enumerate(TEMPERATURES):
        for j, x in enumerate(FRACTIONS):
            for key in ("Hm_fcc", "d_Hm_fcc_dSi", "cp_fcc"):
                out[key][i, j] = gibbs_energy(T, x, key)
            out["Vmfcc"][i, j] = molar_volume(298, T, x, "Vmfcc")
        out["Hm_dia"][i] = gibbs_energy(T, 0.9999, "Hm_dia")
        out["cp_dia"][i] = gibbs_energy(T, 0.9999, "cp_dia")
        out["Vmdia"][i] = molar_volume(298, T, 0.9999, "Vmdia")
    path = os.path.join(HERE, "reference_thermo.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    _ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PF_KKS_REFERENCE")
    if not _ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_CHECKOUT (or set PF_KKS_REFERENCE)")
    main(_ref)
