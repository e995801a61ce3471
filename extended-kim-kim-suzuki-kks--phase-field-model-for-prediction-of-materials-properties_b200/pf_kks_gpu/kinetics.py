"""Host-side kinetics needed at set-up.

The per-attempt kinetics (vacancy relaxation, diffusivity, mobility, Allen-Cahn
coefficient, normalisation; ``pf_kks/kinetics.py:9-107``) run on the device in
``csrc/kks_scalar.cu``, with the constants of ``pf_kks/constants.py:6-21``.
The host only needs the initial vacancy site fraction.
"""

import numpy as np

R = 8.314472
HF1VA = 63680
SF1VA = 2.49
HB = 10613
SB_KB = 42453
Z_COORD = 12


def quenched_vacancy_fraction(T_quench):
    """Vacancy site fraction frozen in from ``T_quench`` (pf_kks/kinetics.py:17-21)."""
    return np.exp(-(HF1VA - T_quench * SF1VA) / (R * T_quench)) * (
        1 - Z_COORD * 0.01 + Z_COORD * 0.01 * np.exp((HB - T_quench * SB_KB) / (R * T_quench))
    )
