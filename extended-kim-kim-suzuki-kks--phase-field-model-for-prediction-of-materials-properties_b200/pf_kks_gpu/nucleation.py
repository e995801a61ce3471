"""Classical nucleation of Si precipitates (optional coupling).

Drop-in for ``pf_kks.nucleation`` (``pf_kks/nucleation.py:15-111``) plus the
device side of the random insertion:

* :func:`nucleation_increment` - expected number of nuclei formed in the box
  during ``dt`` and the critical radius (classical nucleation theory with an
  elastic misfit correction for an incoherent spherical Si precipitate and a
  heterogeneous factor ``B``); scalar host arithmetic, with the elastic
  constants and molar volumes it needs (the fits of ``pf_kks/thermo.py:523-690``);
* :func:`insert_random_nucleus` - the reference's host version, eta = 1 at one
  random candidate;
* :func:`insert_random_nucleus_on_device` - the same on a device cell, with
  the candidates of the original ``put_nucle`` (points with eta < 0.05)
  counted and ranked on the device;
* :class:`NucleationCoupling` - the expected nuclei of each accepted step
  summed from the cell's history rows and inserted between runs.
"""

import math

import numpy as np

N_A = 6.02214086e23  # Avogadro constant [mol^-1] (pf_kks/constants.py:7)
K_B = 1.380649e-23  # Boltzmann constant [J K^-1] (pf_kks/constants.py:8)
X_SI_NUCLEUS = 0.99999  # Si fraction of a nucleus
T_REF_VOLUME = 298.0  # reference temperature of the molar volumes [K]

# Quadratic fits in T of the elastic constants (pf_kks/thermo.py:627-690):
# bulk and Young's moduli of Al [Pa] and C11, C12 of diamond Si [Pa].
_B_AL = (8.030e1 * 1e9, -1.319e-2 * 1e9, -6.815e-6 * 1e9)
_E_AL = (7.028e1 * 1e9, 2.114e-3 * 1e9, -4.903e-5 * 1e9)
_C11_SI = (16.38 * 1e10, -1.28e-3 * 1e10, 0.0)
_C12_SI = (5.92 * 1e10, -0.48e-3 * 1e10, 0.0)

# Integrated thermal-expansion fits (pf_kks/thermo.py:523-625): V0 [m^3/mol] and
# the a, b, c, d coefficients of alpha(T) = (a + b T + c T^2 + d T^-2) / 3.
_VM_FCC_AL = (9.99987596e-6, 2.17303609e-05, 2.63550737e-09, 1.47000588e-11, -9.03030712e-02)
_VM_FCC_SI = (9.20000852e-6, 4.50736462e-06, 2.00632966e-09, -8.07642813e-13, -1.50848370e-01)
_VM_DIA_SI = (1.20588085e-05, 3.43321444e-06, 1.54351184e-09, -6.13087337e-13, -1.14950173e-01)


def _quad(c, T):
    return c[0] + c[1] * T + c[2] * T**2


def elastic_constants(T):
    """C11, C12 of Al (from its bulk and Young's moduli) and of Si, at T [K]
    (the products and quotients in the reference's order, for equal rounding)."""
    B, E = _quad(_B_AL, T), _quad(_E_AL, T)
    return {"C11": B - 4 * E * B / (E - 9 * B), "C12": B + 2 * E * B / (E - 9 * B), "C11_Si": _quad(_C11_SI, T),
            "C12_Si": _quad(_C12_SI, T)}


def _expansion_volume(fit, T0, T):
    V0, a, b, c, d = fit

    def primitive(t):
        return a * t + (b / 2) * t**2 + (c / 3) * t**3 + d * (-(t ** (-1)))

    return V0 * np.exp(3 * (primitive(T) - primitive(T0)))


def molar_volume_fcc(T0, T, X_Si):
    """Molar volume of the FCC phase with Si fraction X_Si [m^3/mol]."""
    return (1 - X_Si) * _expansion_volume(_VM_FCC_AL, T0, T) + X_Si * _expansion_volume(_VM_FCC_SI, T0, T)


def molar_volume_diamond(T0, T):
    """Molar volume of diamond Si [m^3/mol]."""
    return _expansion_volume(_VM_DIA_SI, T0, T)


def nucleation_increment(B, X_al_eq, t, dt, T, dx, dy, dz, nx, ny, nz, D, A_alp, B_alp, C_alp, A_thet, B_thet,
                         C_thet, sigma, X_al_mean, Xv):
    """Expected nuclei formed during ``dt`` in the simulated volume, and the
    critical radius [m] (pf_kks/nucleation.py:15-98). Both are 0 once the
    matrix Si fraction is below ``X_al_eq``; the matrix fraction used in the
    driving force is capped at 0.025."""
    x = 0.025 if X_al_mean > 0.025 else X_al_mean
    el = elastic_constants(T)
    K_si = (el["C11_Si"] + 2 * el["C12_Si"]) / 3
    mu_al = (el["C11"] - el["C12"]) / 2
    c6 = (3 * K_si) / (3 * K_si + 4 * mu_al)

    Vm_fcc = molar_volume_fcc(T_REF_VOLUME, T, x)
    a_fcc = (4 * (Vm_fcc / N_A)) ** (1 / 3)  # 4 atoms per FCC cell
    Vm_dia = molar_volume_diamond(T_REF_VOLUME, T)
    V_dia = Vm_dia / N_A
    Vm = 0.1 * Vm_dia + 0.9 * Vm_fcc

    # simulated volume: the 1-D and 2-D boxes are extended to a cube of the same size
    if ny == 1 and nz == 1:
        Vsim = ((nx - 1) * dx) ** 3
    elif nz == 1:
        Vsim = ((nx - 1) * dx * (ny - 1) * dy) ** (3 / 2)
    else:
        Vsim = (nx - 1) * dx * (ny - 1) * dy * (nz - 1) * dz

    # chemical driving force per atom, with the reference's slope term 2 A x + B x
    slope = 2 * A_alp * x + B_alp * x
    f_nucleus = A_thet * X_SI_NUCLEUS**2 + B_thet * X_SI_NUCLEUS + C_thet
    f_matrix = A_alp * x**2 + B_alp * x + C_alp
    dg_v = (1 / N_A) * (f_nucleus - (f_matrix + slope * (X_SI_NUCLEUS - x)))

    shape = (36 * np.pi * V_dia**2) ** (1 / 3.0)
    misfit = (1 / 3) * ((Vm_dia - Vm_fcc) ** 2 / Vm_dia) / N_A
    dg_s = 2 * mu_al * c6 * misfit
    dg = dg_v + dg_s
    barrier = B * ((4 / 27) * ((shape * sigma) ** 3 / dg**2))

    n_crit = (-2 * shape * sigma / (3 * dg)) ** 3
    r_crit = (1 / (2 * np.sqrt(np.pi))) * (36 * np.pi) ** (1 / 6) * V_dia ** (1 / 3) * n_crit ** (1 / 3)
    zeldovich = (3 * dg**2) / (4 * np.sqrt(np.pi * K_B * T) * (sigma * shape) ** (3 / 2.0))
    attach = (4 * np.pi * r_crit**2 * x * D) / (a_fcc**4)
    incubation = 1 / (2 * attach * zeldovich**2)
    rate = zeldovich * Xv * attach * np.exp(-barrier / (K_B * T)) * np.exp(-incubation / t) * (N_A / Vm) * Vsim

    n_nuclei = rate * dt
    if x < X_al_eq:
        return 0, 0
    return n_nuclei, r_crit


def insert_random_nucleus(candidates, eta, rng=None):
    """eta = 1 at one random point among ``candidates`` (flat indices), on host
    arrays (pf_kks/nucleation.py:103-111). The draw is ``randint(0, n - 1)``,
    as in the reference: the last candidate is never picked."""
    rng = np.random if rng is None else rng
    flat = eta.reshape(-1)
    pick = rng.randint(0, len(candidates) - 1, size=1)
    flat[np.asarray(candidates)[pick]] = 1
    return flat.reshape(eta.shape)


def insert_random_nucleus_on_device(cell, rng=None, eta_below=0.05):
    """:func:`insert_random_nucleus` on the state of a device cell, with the
    candidates ``flatnonzero(eta < eta_below)`` counted and ranked on the
    device (no field leaves the GPU). Returns the candidate rank inserted."""
    rng = np.random if rng is None else rng
    count = cell.count_below(eta_below)
    pick = rng.randint(0, count - 1, size=1)
    cell.insert_nuclei(pick, eta_below)
    return int(pick[0])


class NucleationCoupling:
    """Random nucleation between runs of a device cell.

    After each accepted step the expected number of nuclei of that step
    (:func:`nucleation_increment` at the step's temperature, time step,
    diffusivity, vacancy fraction and matrix Si mean, read from the cell's
    history row; interface energy and parabola coefficients from the material
    tables at that temperature) is added to a running sum; each time the sum
    passes an integer, one nucleus is inserted on the device at a random point
    with eta < ``eta_below``. The nuclei are therefore inserted at the end of
    the ``cell.run`` call whose steps produced them: run one step per call for
    insertion at the step where it occurs.
    """

    def __init__(self, cfg, tables, B, X_al_eq=None, eta_below=0.05, rng=None):
        self.cfg, self.tables, self.B = cfg, tables, B
        self.X_al_eq = cfg.x_equilibrium if X_al_eq is None else X_al_eq
        self.eta_below = eta_below
        self.rng = np.random.RandomState(0) if rng is None else rng
        self.expected = 0.0
        self.inserted = []  # (istep, candidate rank)

    def increment(self, row):
        """Expected nuclei of the step of one history row (``_lib.H`` columns)."""
        from ._lib import H

        T = float(row[H["T"]])
        t_end = float(row[H["time"]]) + float(row[H["dtime"]])
        c = {k: float(self.tables.at(T, k)) for k in ("A_alp", "B_alp", "C_alp", "A_thet", "B_thet", "C_thet")}
        n, _ = nucleation_increment(self.B, self.X_al_eq, t_end, float(row[H["dtime"]]), T, self.cfg.dx,
                                    self.cfg.dx, self.cfg.dx, self.cfg.nx, self.cfg.ny, 1, float(row[H["D"]]),
                                    c["A_alp"], c["B_alp"], c["C_alp"], c["A_thet"], c["B_thet"], c["C_thet"],
                                    float(self.tables.at(T, "gamma")), float(row[H["X_al_mean"]]),
                                    float(row[H["Xv"]]))
        return n if math.isfinite(n) else 0.0

    def after_run(self, cell, rows):
        """Add the expected nuclei of the steps of ``rows`` (history rows of
        the run that just ended) and insert every whole nucleus owed; returns
        the number inserted."""
        from ._lib import H

        istep = -1
        for row in rows:
            self.expected += self.increment(row)
            istep = int(row[H["istep"]])
        done = 0
        while self.expected >= 1.0:
            self.expected -= 1.0
            rank = insert_random_nucleus_on_device(cell, self.rng, self.eta_below)
            self.inserted.append((istep, rank))
            done += 1
        return done
