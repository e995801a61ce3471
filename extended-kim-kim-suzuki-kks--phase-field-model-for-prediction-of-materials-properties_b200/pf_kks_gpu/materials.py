"""Temperature-dependent material tables (``final_export.npz``).

The file is a data format of the reference (``pf_kks/materials.py:33-55``):
six-point tables over T = 400..850 K stored under the names of the CALPHAD
phases (FCC matrix, diamond precipitate). ``NPZ_KEYS`` maps each table of the
step to its key in the file; the two calibration factors scale the interface
energy (``c_gamma``) and the misfit strain (``c_eps0``) at load time, as the
reference does. ``at`` is the host-side linear interpolation (``np.interp``);
the GPU step interpolates the same tables on the device every attempt.
"""

import os
from dataclasses import dataclass

import numpy as np

# Order of the tables in the device parameter block (include/kks.h, KKS_TAB_*).
TABLE_ORDER = ("A_alp", "B_alp", "C_alp", "A_thet", "B_thet", "C_thet", "C11", "C12", "C44", "epsX", "Vm", "gamma",
               "X_Si_fcc")

# table of the step -> key in final_export.npz
NPZ_KEYS = {
    "A_alp": "A_fcc", "B_alp": "B_fcc", "C_alp": "C_fcc",      # matrix parabola A c^2 + B c + C [J/mol]
    "A_thet": "A_dia", "B_thet": "B_dia", "C_thet": "C_dia",   # precipitate parabola [J/mol]
    "C11": "C11", "C12": "C12", "C44": "C44",                  # matrix stiffness [Pa]
    "epsX": "delta",                                           # dilatational misfit [-]
    "Vm": "Vm",                                                # molar volume [m^3/mol]
    "gamma": "gamma",                                          # interface energy [J/m^2]
    "X_Si_fcc": "X_Si_fcc",                                    # matrix equilibrium Si fraction [-]
}

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
DEFAULT_TABLES = os.path.join(DATA_DIR, "final_export.npz")
DEFAULT_PRECIPITATES = os.path.join(DATA_DIR, "micro_final.npz")


@dataclass
class MaterialTables:
    T: np.ndarray
    A_alp: np.ndarray
    B_alp: np.ndarray
    C_alp: np.ndarray
    A_thet: np.ndarray
    B_thet: np.ndarray
    C_thet: np.ndarray
    C11: np.ndarray
    C12: np.ndarray
    C44: np.ndarray
    epsX: np.ndarray
    Vm: np.ndarray
    gamma: np.ndarray
    X_Si_fcc: np.ndarray
    D0: float   # Si diffusion prefactor stored with the tables [m^2/s]
    QD: float   # its activation energy [J/mol]

    @classmethod
    def from_npz(cls, path, c_gamma=1.0, c_eps0=1.0):
        """Read the tables; gamma is multiplied by ``c_gamma`` and epsX by
        ``c_eps0``."""
        scale = {"gamma": c_gamma, "epsX": c_eps0}
        with np.load(path) as d:
            tables = {name: d[key] * scale[name] if name in scale else d[key] for name, key in NPZ_KEYS.items()}
            return cls(T=d["T"], D0=d["D0"], QD=d["QD"], **tables)

    def at(self, T, name):
        return np.interp(T, self.T, getattr(self, name))
