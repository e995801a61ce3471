"""Temperature-dependent material tables (``final_export.npz``).

Same loader semantics as ``pf_kks.materials.MaterialTables.from_npz``
(``pf_kks/materials.py:33-55``): interface energy scaled by ``c_gamma``, misfit
by ``c_eps0``. ``at`` is the host-side ``np.interp``; the GPU step interpolates
the same tables on the device every attempt.
"""

import os
from dataclasses import dataclass

import numpy as np

# Order of the tables in the device parameter block (csrc/kks_abi.h, KKS_TAB_*).
TABLE_ORDER = ("A_alp", "B_alp", "C_alp", "A_thet", "B_thet", "C_thet", "C11", "C12", "C44", "epsX", "Vm", "gamma",
               "X_Si_fcc")

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
    D0: float
    QD: float

    @classmethod
    def from_npz(cls, path, c_gamma=1.0, c_eps0=1.0):
        d = np.load(path)
        return cls(
            T=d["T"],
            A_alp=d["A_fcc"],
            B_alp=d["B_fcc"],
            C_alp=d["C_fcc"],
            A_thet=d["A_dia"],
            B_thet=d["B_dia"],
            C_thet=d["C_dia"],
            C11=d["C11"],
            C12=d["C12"],
            C44=d["C44"],
            epsX=d["delta"] * c_eps0,
            Vm=d["Vm"],
            gamma=d["gamma"] * c_gamma,
            X_Si_fcc=d["X_Si_fcc"],
            D0=d["D0"],
            QD=d["QD"],
        )

    def at(self, T, name):
        return np.interp(T, self.T, getattr(self, name))
