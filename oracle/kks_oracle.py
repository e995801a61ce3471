"""CPU oracle of the extended-KKS semi-implicit FFT time step.

TEST INFRASTRUCTURE ONLY. This module is the checker that the CUDA path is
compared against. Only the test-suite, the smoke check of ``__graft_entry__``
and the CPU-baseline / reference leg of ``bench.py`` may import it; the product
(``pf_kks_gpu``) never does and has no CPU fallback.

It restates, in plain numpy, the time loop of the reference package ``pf_kks``
(``pf_kks/solver.py:76-414``) and the physics functions it calls, each function
citing the reference lines it follows. One deliberate difference: the
Khachaturyan elasticity solve (``pf_kks/elasticity.py:107-163``, with the Green
operator of ``:60-94``) is written in its closed 2-D form. With ``nz = 1`` the
wave vector has no z component, the eigenstrain is dilatational and the total
strain starts at zero, so the 81-component Green-operator contraction reduces to

    eps_hat_kh = epsX (C11 + 2 C12) FT(eta^2) * 0.5 ((N k)_h k_k + (N k)_k k_h)

with ``N`` the inverse of the 2x2 acoustic tensor (zero at k = 0), and

    el_eta = 2 epsX eta (C11 + 2 C12) (3 epsX eta^2 - tr eps)
    el     = 1/2 sigma : eps_el,  eps_el = eps - epsX eta^2 I.

The reduction is exact in real arithmetic; it changes round-off only.

``run(update=...)`` can replace the update by an emulation of the mixed CUDA
step (single-precision transforms; accuracy studies only). The default is the
reference's update, and every pin below is of that default.

Parity of this oracle is PINNED (tests/test_oracle_golden.py):

* against the map the 2022 reproducible run archived after its first step
  (735 x 735; reference test ``tests/test_archived_run.py:35-46``, atol 1e-14)
  and the first 20 archived history rows (``:49-61``, rtol 1e-12);
* against fixtures produced by running ``pf_kks`` itself on the setups of the
  reference's equivalence tests (``tests/test_solver_equivalence.py:79-118``):
  fixed steps, accepted, enlarged, rejected + abort, with byte-identical logs.
"""

import datetime
import os
import time
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# Constants: pf_kks/constants.py:6-21
R = 8.314472
HF1VA = 63680
SF1VA = 2.49
HB = 10613
SB_KB = 42453
Z_COORD = 12
D0_AL = 1.7e-4
Q_AL = 142e3
D0_SI_IN_AL = 3.66e-6
Q_SI_IN_AL = 110958


# ---------------------------------------------------------------------------
# Kinetics: pf_kks/kinetics.py:9-107
def equilibrium_vacancy_fraction(T):
    """pf_kks/kinetics.py:9-14"""
    return np.exp(-(HF1VA - T * SF1VA) / (R * T)) * (
        1 - Z_COORD * 0.01 + Z_COORD * 0.01 * np.exp((HB - T * SB_KB) / (R * T))
    )


def quenched_vacancy_fraction(T_quench):
    """pf_kks/kinetics.py:17-21 (same expression at T_quench)."""
    return equilibrium_vacancy_fraction(T_quench)


def si_diffusivity(T, Xv, Xve, D0, QD, cap):
    """pf_kks/kinetics.py:24-38: vacancy-enhanced Si diffusivity, factor capped
    at ``cap`` and ignored below 1."""
    factor = np.abs(1 + (Xv - Xve) / Xve)
    if factor > cap:
        D = cap * D0 * np.exp(-QD / (R * T))
    else:
        D = factor * D0 * np.exp(-QD / (R * T))
    if factor < 1:
        D = D0 * np.exp(-QD / (R * T))
    return D


def effective_vacancy_diffusivity(T, Xv, Xve):
    """pf_kks/kinetics.py:41-45"""
    D_Al = D0_AL * np.exp(-Q_AL / (R * T))
    D_Si = D0_SI_IN_AL * np.exp(-Q_SI_IN_AL / (R * T))
    return np.abs(1 + (Xv - Xve) / Xve) * (0.03 * D_Si + 0.97 * D_Al)


def interface_mobility(T, Meta0, QMeta):
    """pf_kks/kinetics.py:48-50"""
    return Meta0 * np.exp(-QMeta / (R * T))


def vacancy_relaxation(Xv, Xve, dtime, Deff, Lv2):
    """pf_kks/kinetics.py:53-57"""
    dXv = (1 - np.exp(-dtime * (Deff / Lv2))) * (Xve - Xv)
    return Xv + dXv


def gradient_and_barrier(sigma, lambd, alpha):
    """pf_kks/kinetics.py:60-69"""
    kappa2 = 2 * lambd * sigma * 3 / alpha
    w = (sigma * 3 * alpha) / lambd
    return kappa2, w


def allen_cahn_coefficient(sigma, kappa2, w, Meta, D, A_alp, X_Si_fcc, Omega0):
    """pf_kks/kinetics.py:72-80 (thin-interface corrected L, factor 0.01)."""
    kappa = np.sqrt(kappa2)
    xi = (19 / 30) * (1 / Omega0) * 2 * A_alp * (X_Si_fcc - 0.9999) ** 2
    return (sigma / kappa**2) * (1 / (1 / Meta + kappa * xi / (D * np.sqrt(2 * w)))) * 0.01


def normalize(D, D_0, Meta, Meta_0, C44, dx, sigma, alpha, A_thet, B_thet, C_thet, A_alp, B_alp, C_alp, Omega0, L,
              lambd):
    """pf_kks/kinetics.py:83-107 (lengths in dx, energies in C44, time in dx^2/D_0)."""
    kappa2 = 2 * lambd * sigma * 3 / alpha
    w = (sigma * 3 * alpha) / lambd
    return {
        "L_s": (L * C44 * dx**2) / D_0,
        "kappa2_s": kappa2 / (C44 * dx**2),
        "D_s": D / D_0,
        "Meta_s": Meta / Meta_0,
        "w_s": w / (C44),
        "A_thet_s": A_thet / (C44 * Omega0),
        "B_thet_s": B_thet / (C44 * Omega0),
        "C_thet_s": C_thet / (C44 * Omega0),
        "A_alp_s": A_alp / (C44 * Omega0),
        "B_alp_s": B_alp / (C44 * Omega0),
        "C_alp_s": C_alp / (C44 * Omega0),
    }


# ---------------------------------------------------------------------------
# Material tables: pf_kks/materials.py:33-59
TABLE_KEYS = {
    "A_alp": "A_fcc", "B_alp": "B_fcc", "C_alp": "C_fcc",
    "A_thet": "A_dia", "B_thet": "B_dia", "C_thet": "C_dia",
    "C11": "C11", "C12": "C12", "C44": "C44", "epsX": "delta", "Vm": "Vm",
    "gamma": "gamma", "X_Si_fcc": "X_Si_fcc",
}


class Tables:
    """Tables of ``final_export.npz`` with the c_gamma / c_eps0 scaling
    (pf_kks/materials.py:33-55); ``at`` is np.interp (:57-59)."""

    def __init__(self, path, c_gamma=1.0, c_eps0=1.0):
        d = np.load(path)
        self.T = d["T"]
        self.data = {name: d[key] for name, key in TABLE_KEYS.items()}
        self.data["epsX"] = d["delta"] * c_eps0
        self.data["gamma"] = d["gamma"] * c_gamma
        self.D0 = d["D0"]
        self.QD = d["QD"]

    def at(self, T, name):
        return np.interp(T, self.T, self.data[name])


# ---------------------------------------------------------------------------
# Spectral grid: pf_kks/grid.py:6-50
def frequencies(n, d=1.0):
    """Angular wave numbers; the Nyquist entry of an even axis is left at 0
    (pf_kks/grid.py:6-20)."""
    lin = np.zeros(n)
    if n % 2 == 1:
        half = int((n - 1) / 2.0 + 1)
        lin[:half] = np.arange(0, half, 1) * 2 * np.pi / (n * d)
        lin[half:] = np.arange(int(-(n + 1) / 2.0 + 1), 0, 1) * 2 * np.pi / (n * d)
    else:
        lin[0:int(n / 2.0)] = np.arange(0, int(n / 2.0), 1) * 2 * np.pi / (n * d)
        lin[int(n / 2.0 + 1):] = np.arange(int(-n / 2.0 + 1), 0, 1) * 2 * np.pi / (n * d)
    return lin


def wave_vectors(nx, ny):
    """k (3, nx, ny, 1) and k2 of the solver's dimensionless grid (pf_kks/grid.py:23-50)."""
    k = np.zeros((3, nx, ny, 1))
    k[0] = frequencies(nx)[:, None, None]
    k[1] = frequencies(ny)[None, :, None]
    k2 = k[0] ** 2 + k[1] ** 2 + k[2] ** 2
    return k, k2


# ---------------------------------------------------------------------------
# Free energy: pf_kks/free_energy.py:21-110
def free_energy_terms(c_alpha, c_theta, eta, w_s, A_alp_s, B_alp_s, C_alp_s, A_thet_s, B_thet_s, C_thet_s):
    """pf_kks/free_energy.py:21-71, same operation order."""
    fa_s = A_alp_s * c_alpha**2 + B_alp_s * c_alpha + C_alp_s
    fa_ca_s = 2 * A_alp_s * c_alpha + B_alp_s
    fa_caca_s = 2 * A_alp_s
    ft_s = A_thet_s * c_theta**2 + B_thet_s * c_theta + C_thet_s
    ft_ct_s = 2 * A_thet_s * c_theta + B_thet_s
    ft_ctct_s = 2 * A_thet_s
    h = 3.0 * eta**2 - 2 * eta**3
    h_eta = 6.0 * eta - 6 * eta**2
    g = eta**2 - 2 * eta**3 + eta**4
    g_eta = 2.0 * eta - 6.0 * eta**2 + 4.0 * eta**3
    G_s = (1 - h) * fa_s + h * ft_s + w_s * g
    G_eta_s = -h_eta * (fa_s - ft_s - (c_alpha - c_theta) * fa_ca_s) + w_s * g_eta
    G_cc_s = (ft_ctct_s * fa_caca_s) / ((1 - h) * ft_ctct_s + h * fa_caca_s)
    G_ceta_G_cc = h_eta * (c_alpha - c_theta)
    denom = (1 - h) * ft_ctct_s + h * fa_caca_s
    c_alpha_c = ft_ctct_s / denom
    c_theta_c = fa_caca_s / denom
    fa_c_s = fa_ca_s * c_alpha_c
    ft_c_s = ft_ct_s * c_theta_c
    fa_ca_c_s = 2 * A_alp_s * c_alpha_c
    G_ceta_s = -h_eta * (fa_c_s - ft_c_s - (c_alpha_c - c_theta_c) * fa_ca_s - (c_alpha - c_theta) * fa_ca_c_s)
    return G_s, G_eta_s, G_cc_s, G_ceta_G_cc, G_ceta_s, h_eta, fa_ca_s, ft_ct_s


def phase_compositions(X, eta, A_alp, B_alp, A_thet, B_thet):
    """Closed-form KKS phase compositions with the +/-inf and NaN guards
    (pf_kks/free_energy.py:74-95)."""
    h = 3.0 * eta**2 - 2 * eta**3
    with np.errstate(divide="ignore", invalid="ignore"):
        X_al = (X - h * ((B_alp - B_thet) / (2 * A_thet))) / ((1 - h) + h * (A_alp / A_thet))
    X_al[X_al == np.inf] = 1e-6
    X_al[X_al == -np.inf] = -1e-6
    X_al[np.isnan(X_al)] = 1e-6
    X_th = (A_alp / A_thet) * X_al + (B_alp - B_thet) / (2 * A_thet)
    X_th[X_th == np.inf] = 1e-6
    X_th[X_th == -np.inf] = -1e-6
    X_th[np.isnan(X_th)] = 1e-6
    return X_al, X_th


def total_energy(eta, G, kappa2, el):
    """pf_kks/free_energy.py:98-110: np.gradient returns two components, so G
    and el enter twice."""
    nx, ny = eta.shape[0], eta.shape[1]
    eta = eta.reshape(nx, ny)
    G = G.reshape(nx, ny)
    el = el.reshape(nx, ny)
    return (G + 0.5 * kappa2 * (np.asarray(np.gradient(eta))) ** 2 + el).sum()


# ---------------------------------------------------------------------------
# FFT: pf_kks/fft.py:19-74 (complex transforms over axes 0, 1, 2)
class FFT:
    def __init__(self, workers=None):
        self.workers = workers
        if workers is not None:
            import scipy.fft as sfft

            self._sfft = sfft

    def fft(self, a):
        if self.workers is None:
            return np.fft.fftn(a, axes=(0, 1, 2))
        return self._sfft.fftn(a, axes=(0, 1, 2), workers=self.workers)

    def ifft(self, a):
        if self.workers is None:
            return np.fft.ifftn(a, axes=(0, 1, 2))
        return self._sfft.ifftn(a, axes=(0, 1, 2), workers=self.workers)


# ---------------------------------------------------------------------------
# Elasticity (closed 2-D form of pf_kks/elasticity.py:22-163)
class Elasticity:
    """Khachaturyan one-iteration solve with the stiffness frozen at T0
    (pf_kks/solver.py:152-154), in the reduced form given in the module
    docstring."""

    def __init__(self, k, C11, C12, C44):
        self.C11, self.C12, self.C44 = C11, C12, C44
        kx, ky = k[0], k[1]
        Kxx = C11 * kx**2 + C44 * ky**2
        Kyy = C44 * kx**2 + C11 * ky**2
        Kxy = (C12 + C44) * kx * ky
        det = Kxx * Kyy - Kxy * Kxy
        zero = det == 0
        det = np.where(zero, 1.0, det)
        Nxx = np.where(zero, 0.0, Kyy / det)
        Nyy = np.where(zero, 0.0, Kxx / det)
        Nxy = np.where(zero, 0.0, -Kxy / det)
        Nkx = Nxx * kx + Nxy * ky
        Nky = Nxy * kx + Nyy * ky
        # 0.5 ((N k)_h k_k + (N k)_k k_h) for (k, h) = xx, yy, xy
        self.Oxx = Nkx * kx
        self.Oyy = Nky * ky
        self.Oxy = 0.5 * (Nky * kx + Nkx * ky)

    def solve(self, eta, epsX, fft):
        """Returns sig_el, eps_el (3, 3, nx, ny, 1), el_eta, el
        (pf_kks/elasticity.py:107-163)."""
        C11, C12, C44 = self.C11, self.C12, self.C44
        c3 = C11 + 2 * C12
        A = (epsX * c3) * fft.fft(eta**2)
        exx = np.real(fft.ifft(A * self.Oxx))
        eyy = np.real(fft.ifft(A * self.Oyy))
        exy = np.real(fft.ifft(A * self.Oxy))
        a = epsX * eta**2
        e_xx = exx - a
        e_yy = eyy - a
        e_zz = -a
        s_xx = C11 * e_xx + C12 * (e_yy + e_zz)
        s_yy = C11 * e_yy + C12 * (e_xx + e_zz)
        s_zz = C11 * e_zz + C12 * (e_xx + e_yy)
        s_xy = 2 * C44 * exy
        el = 0.5 * (s_xx * e_xx + s_yy * e_yy + s_zz * e_zz + 2 * s_xy * exy)
        el_eta = 2 * epsX * eta * c3 * (3 * epsX * eta**2 - (exx + eyy))
        nx, ny, nz = eta.shape
        sig = np.zeros((3, 3, nx, ny, nz))
        eps = np.zeros((3, 3, nx, ny, nz))
        sig[0, 0], sig[1, 1], sig[2, 2] = s_xx, s_yy, s_zz
        sig[0, 1] = sig[1, 0] = s_xy
        eps[0, 0], eps[1, 1], eps[2, 2] = e_xx, e_yy, e_zz
        eps[0, 1] = eps[1, 0] = exy
        return sig, eps, el_eta, el


# ---------------------------------------------------------------------------
# Interface measure: pf_kks/microstructure.py:97-128
def interface_area(eta, dx, lambd):
    """Cells (non-periodic, (nx-1)(ny-1)) whose 4 corners satisfy
    0.1 <= eta <= 0.9, times dx^2 / (2 lambd)."""
    if eta.shape[1] == 1:
        return 0
    e = eta[:, :, 0]
    s = (e >= 0.1) & (e <= 0.9)
    cells = s[:-1, :-1] & s[1:, :-1] & s[1:, 1:] & s[:-1, 1:]
    return np.sum(cells) * (dx**2 / (2 * lambd))


# ---------------------------------------------------------------------------
# Residual: pf_kks/residual.py:17-66
@dataclass
class Residual:
    total: float
    energy_derivative: float
    diffusion_term: float
    allen_cahn_term: float
    temperature_term: float


def kks_residual(time_s_history, energy_history, good_step, istep, eta_pair, X_pair, mu_pair, G_pair, L_s, dtime_s):
    """pf_kks/residual.py:26-66"""
    nx, ny = eta_pair[-1].shape[0], eta_pair[-1].shape[1]
    time_s = np.asarray(time_s_history[good_step:])
    energy = energy_history[good_step:istep]
    eta_plus = eta_pair[-1].reshape(nx, ny)
    eta_minus = eta_pair[-2].reshape(nx, ny)
    X_plus = X_pair[-1].reshape(nx, ny)
    X_minus = X_pair[-2].reshape(nx, ny)
    mu_mean = np.asarray((mu_pair[-1].reshape(nx, ny) + mu_pair[-2].reshape(nx, ny)) / 2)
    G = np.asarray(G_pair).reshape(len(G_pair), nx, ny)
    dXdt = (X_plus - X_minus) / dtime_s
    diffusion = dXdt * mu_mean
    energy_derivative = (np.diff(energy) / np.diff(time_s)).mean()
    detadt = (eta_plus - eta_minus) / dtime_s
    allen_cahn = (1 / L_s) * (detadt) ** 2
    temperature = (G[-1] - G[-2]) / dtime_s
    total = energy_derivative + (-1 * diffusion + allen_cahn - temperature).sum()
    return Residual(total, energy_derivative, diffusion.sum(), allen_cahn.sum(), temperature.sum())


# ---------------------------------------------------------------------------
# Run logs: pf_kks/runlog.py:15-140 (the text formats must be identical)
def _e(x):
    return "{0:.2e}".format(x)


class RunLog:
    def __init__(self, directory, enabled=True):
        self.enabled = enabled
        self.log_path = os.path.join(directory, "log.txt")
        self.dtime_path = os.path.join(directory, "dtime.txt")
        if enabled:
            os.makedirs(directory, exist_ok=True)
            with open(self.log_path, "w") as f:
                f.write("start simulation\n")
            with open(self.dtime_path, "w") as f:
                f.write("print time steps\n")

    def _write(self, path, text):
        if self.enabled:
            with open(path, "a") as f:
                f.write(text)

    def state(self, istep, T, D, L, Meta, Omega0, dtime_s):
        self._write(self.dtime_path, "step: " + str(istep) + ", T= " + "{0:.3f} ".format(T) + " D= " + _e(D)
                    + " L= " + _e(L) + " Meta= " + _e(Meta) + " Vm= " + _e(Omega0) + " dtime_s= "
                    + "{0:.2f}".format(dtime_s) + " \n")

    def _terms(self, res, sep_before_temp):
        return ("Residual = " + _e(abs(res.total)) + "," + " Energy_deriv= " + _e(res.energy_derivative) + ","
                + " Potentiel_grad= " + _e(res.diffusion_term) + "," + " eta_term= " + _e(res.allen_cahn_term)
                + sep_before_temp + " temp_term= " + _e(res.temperature_term))

    def rejected(self, istep, iteration, dtime_s, res, energy_s):
        self._write(self.log_path, "step " + str(istep) + ": RE>resmax\n" + self._terms(res, "") + ","
                    + "         Energy= " + _e(energy_s) + "\n")
        self._write(self.dtime_path, "RE>resmax\n" + "repeat istep " + str(istep) + " : iteration " + str(iteration)
                    + " dtime_s:  " + _e(dtime_s) + "\n" + "\n")

    def accepted(self, istep, res, energy_s):
        self._write(self.log_path, "step: " + str(istep) + ", We get  (resmin <RE <resmax) ;  go to step "
                    + str(istep + 1) + "\n" + self._terms(res, ",") + "," + "         Energy= " + _e(energy_s) + "\n")

    def enlarged(self, istep, res, energy_s):
        self._write(self.log_path, " We get  :RE <resmin;  go to step " + str(istep) + "\n" + self._terms(res, ",")
                    + "         Energy= " + _e(energy_s) + "\n")


# ---------------------------------------------------------------------------
# Maps: pf_kks/io.py:20-40
def map_filename(ttime, T_start, T_max):
    return "map" + "{0:.2f}".format(ttime) + "s_" + str(T_start) + "_" + "{0:.2f}".format(T_max) + "K"


def save_map(path, ttime, hist, X, X_al, X_th, eta):
    np.savez_compressed(path, ttime=ttime, time_out=hist["time"], T_out=hist["T"], X_al_mean_out=hist["X_al_mean"],
                        X_th_mean_out=hist["X_th_mean"], eta_mean_out=hist["eta_mean"], surf_out=hist["surf"], X=X,
                        X_al=X_al, X_th=X_th, eta=eta)


# ---------------------------------------------------------------------------
# Time loop: pf_kks/solver.py:40-414
class AdaptiveStepError(RuntimeError):
    """pf_kks/solver.py:72-73"""


@dataclass
class Result:
    X: np.ndarray
    X_al: np.ndarray
    X_th: np.ndarray
    eta: np.ndarray
    sig_el: np.ndarray
    eps_el: np.ndarray
    good_step: int | None
    ttime: float
    map_files: list = field(default_factory=list)
    history: dict = field(default_factory=dict)
    attempts: int = 0
    snapshots: dict = field(default_factory=dict)


HIST_NAMES = ("deta_mean", "eta_mean", "T", "dT", "dtime", "time", "time_s", "surf", "X_al_mean", "X_th_mean",
              "X_mean", "G_mean", "dX_al_mean", "dX_th_mean", "dsurf", "L")


def schedule_steps(cfg):
    """pf_kks/solver.py:46-53: (n_steps, map_steps, surface_steps)."""
    map_steps = np.linspace(1, int(cfg.n_steps), cfg.n_map_saves, dtype=int)
    last = cfg.surface_sample_last_step or cfg.n_steps
    surface_steps = np.linspace(1, int(last), cfg.n_surface_samples, dtype=int)
    return int(np.max(map_steps)), set(map_steps.tolist()), set(surface_steps.tolist())


def _nanmean_masked(a, mask):
    with np.errstate(invalid="ignore", divide="ignore"):
        import warnings

        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            return np.mean(a[mask])


class FFT32:
    """Single-precision transforms (complex64 in, complex64 out) for the
    accuracy studies' emulation of the mixed step; see ``run(update=...)``."""

    def __init__(self):
        import scipy.fft as sfft

        self._sfft = sfft

    def fft(self, a):
        return self._sfft.fftn(np.asarray(a).astype(np.complex64), axes=(0, 1, 2))

    def ifft(self, a):
        return self._sfft.ifftn(np.asarray(a).astype(np.complex64), axes=(0, 1, 2))


def _mixed_update(update, eta, X, drive, G_ceta_G_cc, k, k2, ac_mul, ac_den, ch_mul, bk_mul, fft, fft32):
    """New eta and X of the semi-implicit step (pf_kks/solver.py:249-264) in
    the mixed CUDA step's increment form, for the accuracy studies. With
    a_k = ac_den k^2 and b_k = bk_mul k^2:

        d_eta^ = (ac_mul FT(drive) - a_k FT(eta)) / (1 + a_k)
        d_X^   = (ch_mul FT(flux) - b_k FT(X)) / (1 + b_k),
        flux   = G_ceta_G_cc grad(eta),  grad(eta) = FT^-1(i k FT(eta)),

    transformed back and added to the FP64 state (algebraically the
    reference's update). "mixed": every transform and the spectral arithmetic
    in single precision (drive, flux factor and state rounded to FP32 on
    input), as the mixed CUDA step. "mixed_ch64": the Cahn-Hilliard chain (the
    eta gradients, the flux transforms, FT(X) and d_X^) in FP64, only the
    inverse transform of d_X^ and the Allen-Cahn part in single precision."""
    f32 = np.float32
    k0, k1 = k[0].astype(f32), k[1].astype(f32)
    ak = (ac_den * k2).astype(f32)
    etak32 = fft32.fft(eta)
    d_eta = (f32(ac_mul) * fft32.fft(drive.astype(f32)) - ak * etak32) / (1 + ak)
    eta_b = eta + np.real(fft32.ifft(d_eta)).astype(np.float64)
    if update == "mixed":
        bk = (bk_mul * k2).astype(f32)
        gx = np.real(fft32.ifft(1j * k0 * etak32))
        gy = np.real(fft32.ifft(1j * k1 * etak32))
        gc = G_ceta_G_cc.astype(f32)
        flux_k = 1j * k0 * fft32.fft(gc * gx) + 1j * k1 * fft32.fft(gc * gy)
        d_X = (f32(ch_mul) * flux_k - bk * fft32.fft(X)) / (1 + bk)
    else:
        etak = fft.fft(eta)
        gx = np.real(fft.ifft(1j * k[0] * etak))
        gy = np.real(fft.ifft(1j * k[1] * etak))
        flux_k = 1j * k[0] * fft.fft(G_ceta_G_cc * gx) + 1j * k[1] * fft.fft(G_ceta_G_cc * gy)
        d_X = (ch_mul * flux_k - bk_mul * k2 * fft.fft(X)) / (1 + bk_mul * k2)
    X_b = X + np.real(fft32.ifft(d_X)).astype(np.float64)
    return eta_b, X_b


def run(cfg, eta, X, X_al, X_th, tables_path, out_dir=".", write_logs=True, verbose=False, save_maps=True,
        fft_workers=None, max_steps=None, on_attempt=None, resume=None, snapshot_steps=(), update="fp64"):
    """Restatement of ``pf_kks.solver.run`` (pf_kks/solver.py:76-414).

    ``tables_path`` is the resolved material-table file (the reference resolves
    ``cfg.material_tables`` against ``base_dir``, :102). ``max_steps`` stops the
    loop early (used for bounded CPU-baseline samples); ``on_attempt`` is called
    after each attempt with a dict of the attempt's scalars.

    ``resume`` restarts the loop at a step boundary from a complete loop state
    (the reference itself has no restart): a dict with ``istep`` (the next
    step), the scalars ``flag, good_step, t, t_s, t_b, ttime, Xv, dtime_s, D_0,
    Meta_0, surf, surf_b, T_b`` (``T_b`` None while unset), the per-step
    ``history`` lists of the steps before (at least ``time_s``), ``energy`` and
    ``dtime_s_hist`` arrays of those steps (optionally ``residuals``: the five
    residual-term arrays by name), and, once the adaptive scheme is
    armed, the pair's last entry ``eta_m, X_m, mu_m, G_m`` (pf_kks/solver.py:
    172-173, 353-365). eta, X, X_al, X_th are then the state at ``istep``.
    ``snapshot_steps``: steps at whose start such a dict (plus the four fields
    under ``state``) is recorded in ``Result.snapshots``.

    ``update`` (accuracy studies only): "fp64" is the reference's update;
    "mixed" emulates the mixed CUDA step's increment form with single-precision
    transforms, "mixed_ch64" the same with the Cahn-Hilliard chain in FP64
    (``_mixed_update``). Nothing else changes.
    """
    if update not in ("fp64", "mixed", "mixed_ch64"):
        raise ValueError("update must be fp64, mixed or mixed_ch64")
    t_wall = time.time()
    log = RunLog(out_dir, enabled=write_logs)
    maps_dir = os.path.join(out_dir, "saved_maps")
    if save_maps:
        os.makedirs(maps_dir, exist_ok=True)

    tables = Tables(tables_path, cfg.c_gamma, cfg.c_eps0)
    D0 = (tables.D0 if cfg.D0 is None else cfg.D0) * cfg.c_D
    QD = tables.QD if cfg.QD is None else cfg.QD
    Meta0 = cfg.Meta0 * cfg.c_Meta
    QMeta = cfg.QMeta
    Lv2 = cfg.vacancy_sink_distance**2
    lambd = cfg.half_width_cells * cfg.dx
    alpha = cfg.alpha
    dx = cfg.dx
    nx, ny = cfg.nx, cfg.ny
    time_table = np.array(cfg.schedule_time)
    temp_table = np.array(cfg.schedule_temperature)
    nstep, map_steps, surface_steps = schedule_steps(cfg)
    if max_steps is not None:
        nstep = min(nstep, max_steps)
    fft = FFT(fft_workers)
    fft32 = FFT32() if update != "fp64" else None

    t_s = 0
    t = 0
    t_b = 0
    ttime = 0
    flag = 0
    good_step = None
    hist = {name: [] for name in HIST_NAMES}

    k, k2 = wave_vectors(nx, ny)
    T = np.interp(t, time_table, temp_table)
    elastic = Elasticity(k, tables.at(T, "C11"), tables.at(T, "C12"), tables.at(T, "C44"))

    dtime_s_ini = cfg.dtime_s
    dtime_s = cfg.dtime_s
    dtime_s_min = dtime_s_ini / cfg.dtime_min_divisor
    surf = 0
    surf_b = 0
    T_b = None
    Xv = quenched_vacancy_fraction(cfg.T_quench)

    energy_hist = np.zeros(nstep)
    dtime_s_hist = np.zeros(nstep)
    res_hist = {name: np.zeros(nstep) for name in ("total", "energy_derivative", "diffusion", "allen_cahn",
                                                    "temperature")}
    pair = {name: [] for name in ("mu", "X", "X_al", "X_th", "eta", "D", "G_cc", "G_ceta", "G")}
    num_elem = 2
    map_files = []
    attempts = 0
    sig_el = eps_el = None

    start = 0
    if resume is not None:
        start = int(resume["istep"])
        flag = int(resume["flag"])
        good_step = int(resume["good_step"]) if flag else None
        t, t_s, t_b, ttime = resume["t"], resume["t_s"], resume["t_b"], resume["ttime"]
        Xv, dtime_s = resume["Xv"], resume["dtime_s"]
        D_0, Meta_0 = resume["D_0"], resume["Meta_0"]
        surf, surf_b, T_b = resume["surf"], resume["surf_b"], resume["T_b"]
        for name, values in resume["history"].items():
            hist[name] = list(values)[:start]
        energy_hist[:start] = np.asarray(resume["energy"])[:start]
        dtime_s_hist[:start] = np.asarray(resume["dtime_s_hist"])[:start]
        for name, values in resume.get("residuals", {}).items():
            res_hist[name][:start] = np.asarray(values)[:start]
        if flag:
            for name in pair:
                pair[name] = [None]
            pair["eta"], pair["X"] = [resume["eta_m"]], [resume["X_m"]]
            pair["mu"], pair["G"] = [resume["mu_m"]], [resume["G_m"]]

    snapshots = {}
    for istep in range(start, nstep):
        if istep in snapshot_steps:
            snapshots[istep] = {
                "istep": istep, "flag": flag, "good_step": good_step, "t": t, "t_s": t_s, "t_b": t_b,
                "ttime": ttime, "Xv": Xv, "dtime_s": dtime_s, "D_0": D_0, "Meta_0": Meta_0, "surf": surf,
                "surf_b": surf_b, "T_b": T_b, "history": {k: list(v) for k, v in hist.items()},
                "energy": energy_hist[:istep].copy(), "dtime_s_hist": dtime_s_hist[:istep].copy(),
                "residuals": {k: v[:istep].copy() for k, v in res_hist.items()},
                "state": tuple(np.array(a, copy=True) for a in (eta, X, X_al, X_th)),
            }
            if flag:
                snapshots[istep].update(eta_m=pair["eta"][-1], X_m=pair["X"][-1], mu_m=pair["mu"][-1],
                                        G_m=pair["G"][-1])
        iteration = 1
        while True:
            attempts += 1
            T = np.interp(t, time_table, temp_table)
            if istep + 1 in surface_steps:
                surf = interface_area(eta, dx, lambd)
            Xve = equilibrium_vacancy_fraction(T)
            D = si_diffusivity(T, Xv, Xve, D0, QD, cfg.diffusion_enhancement_cap)
            Meta = interface_mobility(T, Meta0, QMeta)
            Deff = effective_vacancy_diffusivity(T, Xv, Xve)
            if istep == 0:
                D_0 = D
                Meta_0 = Meta
                dtime_s = dtime_s_ini
            if dtime_s > cfg.dtime_max:
                dtime_s = cfg.dtime_max
            if dtime_s < dtime_s_min:
                dtime_s = dtime_s_min
            dtime = (dx**2 / D_0) * dtime_s_ini
            ttime = ttime + dtime
            Xv = vacancy_relaxation(Xv, Xve, dtime, Deff, Lv2)

            A_alp = tables.at(T, "A_alp")
            B_alp = tables.at(T, "B_alp")
            C_alp = tables.at(T, "C_alp")
            C44 = tables.at(T, "C44")
            A_thet = tables.at(T, "A_thet")
            B_thet = tables.at(T, "B_thet")
            C_thet = tables.at(T, "C_thet")
            sigma = tables.at(T, "gamma")
            Omega0 = tables.at(T, "Vm")
            epsX = tables.at(T, "epsX")
            X_Si_fcc = tables.at(T, "X_Si_fcc")
            kappa2, w = gradient_and_barrier(sigma, lambd, alpha)
            L = allen_cahn_coefficient(sigma, kappa2, w, Meta, D, A_alp, X_Si_fcc, Omega0)
            if istep % 100 == 0:
                log.state(istep, T, D, L, Meta, Omega0, dtime_s)
            p = normalize(D, D_0, Meta, Meta_0, C44, dx, sigma, alpha, A_thet, B_thet, C_thet, A_alp, B_alp, C_alp,
                          Omega0, L, lambd)
            coeffs = (p["w_s"], p["A_alp_s"], p["B_alp_s"], p["C_alp_s"], p["A_thet_s"], p["B_thet_s"],
                      p["C_thet_s"])

            G_s, G_eta_s, G_cc_s, G_ceta_G_cc, G_ceta_s, h_eta, fa_ca_s, ft_ct_s = free_energy_terms(
                X_al, X_th, eta, *coeffs)
            sig_el, eps_el, el_eta, el = elastic.solve(eta, epsX, fft)
            el_eta_s = el_eta / C44
            el_s = el / (C44)

            if update == "fp64":
                # Allen-Cahn (pf_kks/solver.py:249-254)
                etak = fft.fft(eta)
                etak_old = etak
                drive_k = fft.fft(G_eta_s + el_eta_s)
                etak = (-dtime_s * p["L_s"] * drive_k + etak) / (1 + dtime_s * p["L_s"] * p["kappa2_s"] * k2)
                eta_b = np.real(fft.ifft(etak))

                # Cahn-Hilliard (pf_kks/solver.py:256-264); the z term is identically zero
                Xk = fft.fft(X)
                flux_k = (1j * k[0] * fft.fft(G_ceta_G_cc * np.real(fft.ifft(1j * k[0] * etak_old)))
                          + 1j * k[1] * fft.fft(G_ceta_G_cc * np.real(fft.ifft(1j * k[1] * etak_old))))
                Xk = (dtime_s * p["D_s"] * flux_k + Xk) / (1 + dtime_s * k2 * p["D_s"])
                X_b = np.real(fft.ifft(Xk))
            else:
                eta_b, X_b = _mixed_update(update, eta, X, G_eta_s + el_eta_s, G_ceta_G_cc, k, k2,
                                           -dtime_s * p["L_s"], dtime_s * p["L_s"] * p["kappa2_s"],
                                           dtime_s * p["D_s"], dtime_s * p["D_s"], fft, fft32)

            # Phase compositions from the start-of-step X (pf_kks/solver.py:266-268)
            X_al_b, X_th_b = phase_compositions(X, eta_b, A_alp, B_alp, A_thet, B_thet)
            energy_s = total_energy(eta_b, G_s, p["kappa2_s"], el_s)
            energy_hist[istep] = energy_s
            dtime_s_hist[istep] = dtime_s
            G_b_s, _, G_cc_b_s, _, G_ceta_b_s, _, fa_ca_s, _ = free_energy_terms(X_al_b, X_th_b, eta_b, *coeffs)

            if flag == 1:
                pair["mu"].append(fa_ca_s)
                pair["X"].append(X_b)
                pair["X_al"].append(X_al_b)
                pair["X_th"].append(X_th_b)
                pair["eta"].append(eta_b)
                pair["D"].append(p["D_s"])
                pair["G_cc"].append(G_cc_b_s)
                pair["G_ceta"].append(G_ceta_b_s)
                pair["G"].append(G_b_s)
            if flag == 1 and istep >= good_step + 1:
                for name in pair:
                    pair[name] = pair[name][-num_elem:]

            info = {"istep": istep, "iteration": iteration, "T": T, "dtime_s": dtime_s, "energy_s": energy_s,
                    "decision": "none"}
            if iteration == cfg.max_iterations:
                raise AdaptiveStepError(
                    f"step {istep}: no admissible time step after {iteration} attempts (dtime_s={dtime_s:.2e})")
            if flag == 0 or istep < good_step + num_elem:
                if on_attempt is not None:
                    on_attempt(info)
                break

            res = kks_residual(hist["time_s"], energy_hist, good_step, istep, pair["eta"], pair["X"], pair["mu"],
                               pair["G"], p["L_s"], dtime_s)
            if not np.isfinite(res.total):
                raise AdaptiveStepError(f"step {istep}: non-finite energy residual")
            res_hist["total"][istep] = res.total
            res_hist["energy_derivative"][istep] = res.energy_derivative
            res_hist["diffusion"][istep] = res.diffusion_term
            res_hist["allen_cahn"][istep] = res.allen_cahn_term
            res_hist["temperature"][istep] = res.temperature_term
            info["residual"] = res
            if verbose and istep % 1000 == 0:
                print("step, |RES-KKS|  , energy_term , gradient_term, eta_term, temp_term : ", istep,
                      "{0:.2e}".format(np.abs(res.total)), "{0:.2e}".format(res.energy_derivative),
                      "{0:.2e}".format(res.diffusion_term), "{0:.2e}".format(res.allen_cahn_term),
                      "{0:.2e}".format(res.temperature_term))
            if np.abs(res.total) > cfg.residual_max:
                dtime_s /= cfg.step_factor
                log.rejected(istep, iteration, dtime_s, res, energy_s)
                info["decision"] = "rejected"
                if on_attempt is not None:
                    on_attempt(info)
                iteration += 1
                continue
            elif np.abs(res.total) > cfg.residual_min:
                log.accepted(istep, res, energy_s)
                info["decision"] = "accepted"
                if on_attempt is not None:
                    on_attempt(info)
                break
            else:
                log.enlarged(istep, res, energy_s)
                dtime_s *= cfg.step_factor
                info["decision"] = "enlarged"
                if on_attempt is not None:
                    on_attempt(info)
                break

        if flag == 1:
            pair["X"][-1] = X_b
            pair["X_al"][-1] = X_al_b
            pair["X_th"][-1] = X_th_b
            pair["eta"][-1] = eta_b
            pair["D"][-1] = p["D_s"]
            pair["G_cc"][-1] = G_cc_s
            pair["G_ceta"][-1] = G_ceta_s
            pair["G"][-1] = G_s
            energy_hist[istep] = energy_s
            dtime_s_hist[istep] = dtime_s

        t_s += dtime_s
        dtime = (dx**2 / D_0) * dtime_s
        t_b += (dx**2 / D_0) * dtime_s
        if istep + 1 in surface_steps:
            T_b = np.interp(t_b, time_table, temp_table)
            surf_b = interface_area(eta_b, dx, lambd)

        X_al_mean = _nanmean_masked(X, eta < 0.05)
        if X_al_mean <= cfg.x_equilibrium and flag == 0 and istep > 1:
            good_step = istep + cfg.good_step_offset
            flag = 1

        hist["X_al_mean"].append(X_al_mean)
        hist["X_th_mean"].append(_nanmean_masked(X, eta > 0.95))
        hist["X_mean"].append(_nanmean_masked(X, (eta > 0.05) & (eta > 0.95)))
        hist["dX_al_mean"].append(_nanmean_masked(X_b, eta_b < 0.05) - _nanmean_masked(X, eta < 0.05))
        hist["dX_th_mean"].append(_nanmean_masked(X_b, eta_b > 0.95) - _nanmean_masked(X, eta > 0.95))
        hist["deta_mean"].append(np.mean(eta_b) - np.mean(eta))
        hist["dT"].append(T_b - T)
        hist["eta_mean"].append(np.mean(eta))
        hist["G_mean"].append(np.mean(G_s.reshape(nx, ny)))
        hist["surf"].append(surf_b)
        hist["dsurf"].append(surf_b - surf)
        hist["T"].append(T)
        hist["dtime"].append(dtime)
        hist["time"].append(t)
        hist["time_s"].append(t_s)
        hist["L"].append(L)

        eta, X, X_al, X_th = eta_b, X_b, X_al_b, X_th_b
        t = t_b

        if save_maps and istep + 1 in map_steps:
            name = map_filename(ttime, cfg.schedule_temperature[0], np.asarray(hist["T"]).max())
            path = os.path.join(maps_dir, name)
            save_map(path, ttime, hist, X, X_al, X_th, eta)
            map_files.append(path + ".npz")

    if verbose:
        print("Temperature reached : %s K ---" % (np.asarray(hist["T"]).max()))
        print("simulation time : " + str(datetime.timedelta(seconds=time.time() - t_wall)))

    hist["energy_s"] = energy_hist
    hist["dtime_s"] = dtime_s_hist
    for name, values in res_hist.items():
        hist["residual_" + name] = values
    return Result(X, X_al, X_th, eta, sig_el, eps_el, good_step, ttime, map_files, hist, attempts, snapshots)
