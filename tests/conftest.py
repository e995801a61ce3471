"""Shared test set-up.

* ``gpu`` marks tests that need a CUDA device (run with ``-m gpu``); every other
  test runs on the CPU.
* The package directory is put on ``sys.path`` so that ``pf_kks_gpu`` and the
  ``oracle`` package import from the checkout.
"""

import os
import re
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "extended-kim-kim-suzuki-kks--phase-field-model-for-prediction-of-materials-properties_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (PKG, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

from pf_kks_gpu.config import SimulationConfig  # noqa: E402
from pf_kks_gpu.materials import DEFAULT_TABLES  # noqa: E402
from pf_kks_gpu.microstructure import place_precipitates  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def small_config(**overrides):
    """64 x 64 grid with the reproducible-run parameters (the reference's
    tests/conftest.py:19-30 set-up)."""
    params = dict(nx=64, ny=64, n_steps=40, n_map_saves=3, n_surface_samples=10, material_tables=DEFAULT_TABLES)
    params.update(overrides)
    return SimulationConfig(**params)


def three_precipitates(cfg):
    """Three sharp precipitates (the reference's tests/conftest.py:33-39)."""
    dx = cfg.dx
    r = np.array([3e-9, 2e-9, 4e-9])
    ox = np.array([8e-9, 20e-9, cfg.nx * dx * 0.6])
    oy = np.array([10e-9, 22e-9, cfg.ny * dx * 0.3])
    return place_precipitates(cfg.nx, cfg.ny, cfg.nz, dx, dx, dx, cfg.x_matrix, cfg.x_precipitate, r, ox, oy,
                              np.zeros(3))


def copy_state(state):
    return tuple(np.array(a, copy=True) for a in state)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


_NUM = re.compile(r"[-+]?\d+\.\d+(?:e[-+]\d+)?|[-+]?\d+")


def assert_logs_equivalent(a, b, tiny=1e-8, tiny_rtol=0.05, zero=1e-15):
    """Logs with the same lines and decisions: the text around the numbers is
    identical, integers are equal, and reals agree within one unit of their
    last printed digit (the log prints 3 significant digits). Reals below
    ``tiny`` in magnitude (residual terms at round-off level) may differ by
    ``tiny_rtol`` relative, and reals below ``zero`` on both sides (sums of
    differences of identical states: pure round-off) count as equal."""
    la, lb = a.splitlines(), b.splitlines()
    assert len(la) == len(lb), (len(la), len(lb))
    for x, y in zip(la, lb):
        assert _NUM.sub("#", x) == _NUM.sub("#", y), (x, y)
        for u, v in zip(_NUM.findall(x), _NUM.findall(y)):
            if "." not in u:
                assert u == v, (x, y)
                continue
            fu, fv = float(u), float(v)
            if max(abs(fu), abs(fv)) < zero:
                continue
            if "e" in u:
                ulp = 10.0 ** (int(u.split("e")[1]) - 2)
            else:
                ulp = 10.0 ** -len(u.split(".")[1])
            tol = 1.0001 * ulp
            if abs(fv) < tiny:
                tol = max(tol, tiny_rtol * abs(fv))
            assert abs(fu - fv) <= tol, (x, y)


@pytest.fixture(scope="session")
def small_golden():
    return np.load(os.path.join(GOLDEN, "reference_small.npz"))


@pytest.fixture(scope="session")
def small_golden_logs():
    import json

    with open(os.path.join(GOLDEN, "reference_small_logs.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def relaxed_state(small_golden):
    """The reference's relaxed_state fixture (300 unarmed steps), as computed by
    pf_kks and stored in the golden fixtures."""
    g = small_golden
    return tuple(np.array(g[f"relaxed_{k}"]) for k in ("eta", "X", "X_al", "X_th"))


def gpu_loop_state(cell, rows):
    """The loop state of a GPU cell at its current step boundary, in the form
    the oracle's ``resume`` takes, and the current fields. ``rows`` are all the
    history rows the cell produced so far (one per step, from ``drain``)."""
    from pf_kks_gpu import _lib as L
    from pf_kks_gpu.solver import HIST_NAMES

    s = cell.state()
    rows = np.asarray(rows)
    assert rows.shape[0] == s.istep
    H = L.H
    hist = {name: [float(v) for v in rows[:, H[name]]] for name in HIST_NAMES}
    if s.istep:
        hist["time"][0] = 0
    resume = {
        "istep": int(s.istep), "flag": int(s.flag), "good_step": int(s.good_step), "t": s.t, "t_s": s.t_s,
        "t_b": s.t_b, "ttime": s.ttime, "Xv": s.Xv, "dtime_s": s.dtime_s, "D_0": s.D_0, "Meta_0": s.Meta_0,
        "surf": s.surf, "surf_b": s.surf_b, "T_b": s.T_b, "history": hist,
        "energy": rows[:, H["energy_s"]].copy(), "dtime_s_hist": rows[:, H["dtime_s"]].copy(),
        "residuals": {name: rows[:, H["residual_" + name]].copy()
                      for name in ("total", "energy_derivative", "diffusion", "allen_cahn", "temperature")},
    }
    if s.flag:
        resume["eta_m"], resume["X_m"], resume["mu_m"], resume["G_m"] = cell.download_pair()
    return resume, cell.download()
