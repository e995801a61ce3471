"""A pure-torch float64 restatement of one fixed-dt step (test infrastructure:
the autograd reference for the hand-written adjoint of ``csrc/kks_adjoint.cu``).

Same operations as the oracle's attempt with ``flag == 0``
(``oracle/kks_oracle.py`` run loop; ``pf_kks/solver.py:242-268``):
free-energy terms of the old state, the closed 2-D elasticity, the
semi-implicit Allen-Cahn and Cahn-Hilliard updates with the reference's wave
vectors, and the phase compositions of (X_old, eta_b) without the inf / NaN
guards.
"""

import numpy as np
import torch


def wave_numbers(n):
    lin = np.zeros(n)
    if n % 2 == 1:
        half = int((n - 1) / 2.0 + 1)
        lin[:half] = np.arange(half) * 2 * np.pi / n
        lin[half:] = np.arange(int(-(n + 1) / 2.0 + 1), 0) * 2 * np.pi / n
    else:
        lin[: n // 2] = np.arange(n // 2) * 2 * np.pi / n
        lin[n // 2 + 1:] = np.arange(-n // 2 + 1, 0) * 2 * np.pi / n
    return lin


class TorchStep:
    def __init__(self, nx, ny, C11_0, C12_0, C44_0, device="cpu"):
        kx = torch.tensor(wave_numbers(nx), dtype=torch.float64, device=device)[:, None]
        ky = torch.tensor(wave_numbers(ny), dtype=torch.float64, device=device)[None, :]
        self.kx, self.ky = kx.expand(nx, ny), ky.expand(nx, ny)
        self.k2 = self.kx**2 + self.ky**2
        c11, c12 = C11_0 / C44_0, C12_0 / C44_0
        Kxx = c11 * self.kx**2 + self.ky**2
        Kyy = self.kx**2 + c11 * self.ky**2
        Kxy = (c12 + 1) * self.kx * self.ky
        det = Kxx * Kyy - Kxy * Kxy
        zero = det == 0
        det = torch.where(zero, torch.ones_like(det), det)
        Nxx = torch.where(zero, 0 * det, Kyy / det)
        Nyy = torch.where(zero, 0 * det, Kxx / det)
        Nxy = torch.where(zero, 0 * det, -Kxy / det)
        self.otr = (Nxx * self.kx + Nxy * self.ky) * self.kx + (Nxy * self.kx + Nyy * self.ky) * self.ky
        self.cc = C11_0 + 2 * C12_0
        self.c3n = self.cc / C44_0

    def __call__(self, state, c):
        """state: (4, nx, ny) float64; c: 15 coefficients (KKS_COEF_* order)."""
        e, X, ca, ct = state[0], state[1], state[2], state[3]
        dt, Ls, kap, Ds, w, Aa, Ba, Ca, At, Bt, Ct, epsX, C44, pcs, pcr = [c[i] for i in range(15)]
        fft, ifft = torch.fft.fft2, torch.fft.ifft2
        fa = Aa * ca**2 + Ba * ca + Ca
        fa1 = 2 * Aa * ca + Ba
        ft = At * ct**2 + Bt * ct + Ct
        h1 = 6.0 * e - 6 * e**2
        g1 = 2.0 * e - 6.0 * e**2 + 4.0 * e**3
        Geta = -h1 * (fa - ft - (ca - ct) * fa1) + w * g1
        tr = torch.real(ifft(epsX * self.c3n * self.otr * fft(e**2)))
        el = 2 * epsX * e * self.cc * (3 * epsX * e**2 - tr) / C44
        drive = Geta + el
        ek = fft(e)
        p = dt * Ls
        ekb = (-p * fft(drive) + ek) / (1 + p * kap * self.k2)
        eb = torch.real(ifft(ekb))
        gx = torch.real(ifft(1j * self.kx * ek))
        gy = torch.real(ifft(1j * self.ky * ek))
        fl = h1 * (ca - ct)
        flux_k = 1j * self.kx * fft(fl * gx) + 1j * self.ky * fft(fl * gy)
        q = dt * Ds
        Xkb = (q * flux_k + fft(X)) / (1 + q * self.k2)
        Xb = torch.real(ifft(Xkb))
        hb = 3.0 * eb**2 - 2 * eb**3
        cab = (X - hb * pcs) / ((1 - hb) + hb * pcr)
        ctb = pcr * cab + pcs
        return torch.stack([eb, Xb, cab, ctb])
