"""Simulated DSC of a run, differentiable in its histories.

The reference's simulated DSC (``pf_kks/postprocess/dsc.py:78-130``) splits the
apparent heat capacity of the sample into a heat-capacity background, the
precipitation / matrix-desaturation enthalpy and the interface-energy release,
from the histories <eta> (precipitate fraction), <X_Si> of the matrix and the
interface measure. It evaluates the enthalpies, heat capacities and molar
volumes of the FCC matrix and the diamond precipitate with its CALPHAD
description (``pf_kks/thermo.py:147-622``), and the rates from cubic
smoothing splines of the histories sub-sampled every 90 steps.

Here the same three terms are written with forward differences of the
per-step histories (a gradient of a loss over a few hundred steps needs every
step; splines of 90-step samples would leave a handful of points), and the
thermodynamic functions are restated in float64 torch so that gradients flow
through the matrix composition:

* pure-element Gibbs energies G0(T) = a + b T + c T ln T + d T^2 + e T^3 + f / T
  of FCC Al (two temperature ranges, split at 700 K) and diamond Si (up to
  1687 K), the SGTE unary data; the lattice-stability offsets of FCC Si and
  diamond Al and the regular-solution parameters L0(T) of the two phases, the
  COST 507 Al-Si assessment; the same numbers as the reference's description.
  Enthalpy H = G - T dG/dT and heat capacity cp = -T d2G/dT2 are taken
  analytically from that form (the ideal-mixing term R T sum x ln x drops out of
  H exactly, and out of dH/dx);
* molar volumes V0 exp(3 int_T0^T alpha), alpha = (a + b T + c T^2 + d T^-2) / 3,
  of the same thermal-expansion fits, referred to T0 = 298 K.

The restatement is checked against ``pf_kks.thermo.gibbs_energy`` /
``molar_volume`` values on a (T, x) grid (tests/golden/make_thermo_fixture.py).
Valid for 298.15 K < T <= 933.47 K (solid FCC Al), which covers the heat
treatments of the study.
"""

from dataclasses import dataclass

import numpy as np

R_GAS = 8.314472
M_AL, M_SI = 26.98154, 28.0855  # molar masses [g/mol]
X_DIA = 0.9999                  # Si fraction of the precipitate in the reference's DSC

# G0(T) = a + b T + c T ln T + d T^2 + e T^3 + f / T  [J/mol]
_G0_FCC_AL_LOW = (-7976.15, 137.093038, -24.3671976, -1.884662e-3, -0.877664e-6, 74092.0)    # 298.15 < T <= 700
_G0_FCC_AL_HIGH = (-11276.24, 223.048446, -38.5844296, 18.531982e-3, -5.764227e-6, 74092.0)  # 700 < T <= 933.47
_G0_DIA_SI = (-8162.609, 137.236859, -22.8317533, -1.912904e-3, -0.003552e-6, 176667.0)      # 298.15 < T <= 1687
_T_SPLIT_AL = 700.0
# lattice stabilities: G0_fcc_Si = G0_dia_Si + 51000 - 21.8 T, G0_dia_Al = G0_fcc_Al + 30 T
_FCC_SI_OFFSET = (51000.0, -21.8)
_DIA_AL_OFFSET = (0.0, 30.0)
# regular-solution parameters L0 = p + q T
_L0_FCC = (-3143.78, 0.3929)
_L0_DIA = (113246.16, -47.5551)

# thermal-expansion fits (V0 [m^3/mol], a, b, c, d)
_VM_FCC_AL = (9.99987596e-6, 2.17303609e-05, 2.63550737e-09, 1.47000588e-11, -9.03030712e-02)
_VM_FCC_SI = (9.20000852e-6, 4.50736462e-06, 2.00632966e-09, -8.07642813e-13, -1.50848370e-01)
_VM_DIA_SI = (1.20588085e-05, 3.43321444e-06, 1.54351184e-09, -6.13087337e-13, -1.14950173e-01)
T_REF_VOLUME = 298.0


def _torch():
    import torch

    return torch


def _g0_terms(T, coeffs):
    """(G0, H0, d2G0/dT2) of one SGTE range at T (tensor)."""
    torch = _torch()
    a, b, c, d, e, f = coeffs
    lnT = torch.log(T)
    G = a + b * T + c * T * lnT + d * T**2 + e * T**3 + f / T
    dG = b + c * (1 + lnT) + 2 * d * T + 3 * e * T**2 - f / T**2
    d2G = c / T + 2 * d + 6 * e * T + 2 * f / T**3
    return G, G - T * dG, d2G


def _fcc_al(T):
    torch = _torch()
    lo = _g0_terms(T, _G0_FCC_AL_LOW)
    hi = _g0_terms(T, _G0_FCC_AL_HIGH)
    return tuple(torch.where(T <= _T_SPLIT_AL, u, v) for u, v in zip(lo, hi))


def _with_offset(terms, T, offset):
    """(G, H, d2G/dT2) of G0 + p + q T: H gains p, d2G is unchanged."""
    G, H, d2G = terms
    p, q = offset
    return G + p + q * T, H + p, d2G


def _l0(T, par):
    """(L0, L0 - T dL0/dT) of a linear L0 = p + q T."""
    p, q = par
    return p + q * T, p + 0 * T


@dataclass
class PhaseThermo:
    """Thermodynamic functions of the two phases at (T, x) (tensors)."""

    Hm_fcc: object       # molar enthalpy of the FCC matrix at Si fraction x [J/mol]
    dHm_fcc_dx: object   # its derivative with respect to x
    cp_fcc: object       # heat capacity of the matrix [J/(mol K)]
    Hm_dia: object       # molar enthalpy of the diamond precipitate (x = 0.9999)
    cp_dia: object
    Vm_fcc: object       # molar volumes [m^3/mol]
    Vm_dia: object


def _expansion_volume(T, fit, T0=T_REF_VOLUME):
    torch = _torch()
    V0, a, b, c, d = fit

    def primitive(t):
        return a * t + (b / 2) * t**2 + (c / 3) * t**3 - d / t

    return V0 * torch.exp(3 * (primitive(T) - primitive(T0 + 0 * T)))


def phase_thermo(T, x):
    """Enthalpies, heat capacities and molar volumes of the FCC matrix (Si
    fraction x) and of the diamond precipitate at temperature T; T and x are
    float64 tensors of one shape, and every output is differentiable in both."""
    al_fcc = _fcc_al(T)
    si_dia = _g0_terms(T, _G0_DIA_SI)
    si_fcc = _with_offset(si_dia, T, _FCC_SI_OFFSET)
    al_dia = _with_offset(al_fcc, T, _DIA_AL_OFFSET)
    _, hl_fcc = _l0(T, _L0_FCC)
    _, hl_dia = _l0(T, _L0_DIA)
    xd = X_DIA + 0 * T
    Hm_fcc = (1 - x) * al_fcc[1] + x * si_fcc[1] + x * (1 - x) * hl_fcc
    dHm_fcc_dx = si_fcc[1] - al_fcc[1] + (1 - 2 * x) * hl_fcc
    cp_fcc = -T * ((1 - x) * al_fcc[2] + x * si_fcc[2])
    Hm_dia = (1 - xd) * al_dia[1] + xd * si_dia[1] + xd * (1 - xd) * hl_dia
    cp_dia = -T * ((1 - xd) * al_dia[2] + xd * si_dia[2])
    Vm_fcc = (1 - x) * _expansion_volume(T, _VM_FCC_AL) + x * _expansion_volume(T, _VM_FCC_SI)
    Vm_dia = _expansion_volume(T, _VM_DIA_SI)
    return PhaseThermo(Hm_fcc, dHm_fcc_dx, cp_fcc, Hm_dia, cp_dia, Vm_fcc, Vm_dia)


@dataclass
class DSCParameters:
    """Parameters of the simulated DSC, with the reference's defaults
    (``pf_kks/postprocess/dsc.py:28-39``) except the simulated area, which is
    the cell's own (nx dx)^2 / 4 when built by :meth:`for_config`."""

    heating_rate: float = 20 / 60          # K/s
    interface_energy: float = 0.5          # J/m^2
    simulated_area: float = (710e-9) ** 2 / 4
    output_scale: float = 3.0

    @classmethod
    def for_config(cls, cfg, heating_rate=None):
        sched_t = np.asarray(cfg.schedule_time, float)
        sched_T = np.asarray(cfg.schedule_temperature, float)
        if heating_rate is None:
            span = sched_t[-1] - sched_t[0]
            heating_rate = (sched_T[-1] - sched_T[0]) / span if span > 0 else 20 / 60
        return cls(heating_rate=float(heating_rate), simulated_area=(cfg.nx * cfg.dx) ** 2 / 4,
                   output_scale=1.0 / float(heating_rate))


@dataclass
class SimulatedDSC:
    """Per-step DSC terms (one value per forward difference, steps 0..n-2)."""

    T: object
    background: object
    precipitation: object
    surface: object
    scale: float

    @property
    def total(self):
        """Apparent heat capacity Cp* [J/(g K)]."""
        return (self.background + self.precipitation + self.surface) * self.scale


def simulated_dsc(eta_mean, X_al_mean, surf, time, T, params=None):
    """The three DSC terms of ``pf_kks/postprocess/dsc.py:121-130`` from the
    per-step histories, with forward differences for the rates:

        f = <eta>, x = matrix <X_Si>, dt_n = time_{n+1} - time_n
        rho_n        = f_n M_Si / Vm_dia + (1 - f_n) M_Al / Vm_fcc(x_n)
        background_n = rate (f_n cp_dia / M_Si + (1 - f_n) cp_fcc(x_n) / M_Al)
        surface_n    = gamma_H (surf_{n+1} - surf_n) / dt_n / (A_sim rho_n)
        precip._n    = (1 - f_n) dHm_fcc/dx(x_n) / M_Al (x_{n+1} - x_n) / dt_n
                       + (f_{n+1} - f_n) / dt_n (Hm_dia / M_Si - Hm_fcc(x_n) / M_Al)

    all thermodynamic functions at T_n. Inputs are float64 tensors (``surf``
    may be a constant: it has no gradient in a run). Returns SimulatedDSC."""
    torch = _torch()
    p = DSCParameters() if params is None else params
    f, x = eta_mean, X_al_mean
    like = dict(dtype=f.dtype, device=f.device)
    t = torch.as_tensor(time, **like)
    TT = torch.as_tensor(T, **like)
    s = torch.as_tensor(surf, **like)
    dt = t[1:] - t[:-1]
    fn, xn, Tn = f[:-1], x[:-1], TT[:-1]
    th = phase_thermo(Tn, xn)
    rho = fn * M_SI / th.Vm_dia + (1 - fn) * M_AL / th.Vm_fcc
    background = p.heating_rate * (fn * th.cp_dia / M_SI + (1 - fn) * th.cp_fcc / M_AL)
    surface = p.interface_energy * (s[1:] - s[:-1]) / dt / (p.simulated_area * rho)
    precipitation = ((1 - fn) * th.dHm_fcc_dx / M_AL * (x[1:] - xn) / dt
                     + (f[1:] - fn) / dt * (th.Hm_dia / M_SI - th.Hm_fcc / M_AL))
    return SimulatedDSC(Tn, background, precipitation, surface, p.output_scale)
