"""The CPU oracle against the reference's golden data (no GPU).

* the map archived by the 2022 reproducible run after its first step (735^2)
  and its first 20 history rows (the reference's tests/test_archived_run.py);
* pf_kks run here on the set-ups of the reference's equivalence tests
  (tests/test_solver_equivalence.py:79-118): fixed steps, accepted, enlarged,
  rejected + abort, with byte-identical logs;
* pf_kks on the 160^2 synthetic microstructure of this package's generator.
"""

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, copy_state, small_config, three_precipitates

from oracle import kks_oracle
from pf_kks_gpu.config import SimulationConfig
from pf_kks_gpu.materials import DEFAULT_PRECIPITATES, DEFAULT_TABLES
from pf_kks_gpu.microstructure import load_precipitates, place_precipitates

FIELDS = ("X", "X_al", "X_th", "eta")
HIST = ("eta_mean", "deta_mean", "X_mean", "X_al_mean", "dX_al_mean", "X_th_mean", "dX_th_mean", "dT", "T",
        "dtime", "time", "time_s", "surf", "dsurf", "L", "energy_s", "dtime_s", "residual_total",
        "residual_energy_derivative", "residual_diffusion", "residual_allen_cahn", "residual_temperature")


@pytest.mark.parametrize("n", [7, 8, 735])
def test_wave_numbers_match_fft_frequencies(n):
    """pf_kks/grid.py:6-20: 2 pi fftfreq with the Nyquist entry left at 0."""
    expected = 2 * np.pi * np.fft.fftfreq(n)
    if n % 2 == 0:
        expected[n // 2] = 0.0
    np.testing.assert_allclose(kks_oracle.frequencies(n), expected, atol=1e-12)


def test_kks_conditions_hold():
    """Mixture rule and equal diffusion potential (reference tests/test_components.py:35-44)."""
    t = kks_oracle.Tables(DEFAULT_TABLES)
    T = 520.0
    A_a, B_a, A_t, B_t = (t.at(T, n) for n in ("A_alp", "B_alp", "A_thet", "B_thet"))
    eta = np.linspace(0, 1, 11).reshape(11, 1, 1)
    X = np.full_like(eta, 0.3)
    X_al, X_th = kks_oracle.phase_compositions(X, eta, A_a, B_a, A_t, B_t)
    h = 3 * eta**2 - 2 * eta**3
    np.testing.assert_allclose((1 - h) * X_al + h * X_th, X, rtol=1e-12)
    np.testing.assert_allclose(2 * A_a * X_al + B_a, 2 * A_t * X_th + B_t, rtol=1e-9)


def test_drive_vanishes_in_bulk():
    c = np.array([0.01, 0.02])
    for eta in (0.0, 1.0):
        _, G_eta, *_ = kks_oracle.free_energy_terms(c, c + 0.9, np.full(2, eta), 1.0, 2.0, -1.0, 0.1, 3.0, -2.0, 0.5)
        np.testing.assert_array_equal(G_eta, 0.0)


def test_placer_matches_reference(small_golden):
    cfg = small_config()
    eta, X, X_mat, X_pre = three_precipitates(cfg)
    np.testing.assert_array_equal(eta, small_golden["three_init_eta"])
    np.testing.assert_array_equal(X, small_golden["three_init_X"])
    np.testing.assert_array_equal(X_mat, small_golden["three_init_X_al"])
    np.testing.assert_array_equal(X_pre, small_golden["three_init_X_th"])


def _run(cfg, state, out_dir):
    try:
        return kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(out_dir))
    except kks_oracle.AdaptiveStepError as exc:
        return exc


def _check_case(case, res, out_dir, g, logs, field_atol=1e-13, hist_rtol=1e-9):
    for name in FIELDS:
        np.testing.assert_allclose(getattr(res, name), g[f"{case}_{name}"], rtol=0, atol=field_atol, err_msg=name)
    for name in HIST:
        np.testing.assert_allclose(np.asarray(res.history[name], float), g[f"{case}_h_{name}"], rtol=hist_rtol,
                                   atol=1e-14, equal_nan=True, err_msg=name)
    assert (-1 if res.good_step is None else res.good_step) == int(g[f"{case}_good_step"])
    for name in ("log.txt", "dtime.txt"):
        assert (out_dir / name).read_text() == logs[case][name], name
    assert sorted(os.listdir(out_dir / "saved_maps")) == logs[case]["maps"]


def test_fixed_steps(tmp_path, small_golden, small_golden_logs):
    cfg = small_config(n_steps=40)
    res = _run(cfg, three_precipitates(cfg), tmp_path)
    _check_case("fixed40", res, tmp_path, small_golden, small_golden_logs)
    np.testing.assert_allclose(res.sig_el, small_golden["fixed40_sig_el"], rtol=1e-10, atol=1e-3)
    np.testing.assert_allclose(res.eps_el, small_golden["fixed40_eps_el"], rtol=0, atol=1e-14)


def test_accepted_steps(tmp_path, relaxed_state, small_golden, small_golden_logs):
    cfg = small_config(n_steps=30, x_equilibrium=0.2)
    res = _run(cfg, relaxed_state, tmp_path)
    _check_case("accepted30", res, tmp_path, small_golden, small_golden_logs)
    assert res.good_step == 2


def test_enlarged_steps(tmp_path, relaxed_state, small_golden, small_golden_logs):
    cfg = small_config(n_steps=40, x_equilibrium=0.2, dtime_s=60, dtime_max=150, residual_min=7.6e-4)
    res = _run(cfg, relaxed_state, tmp_path)
    _check_case("enlarged40", res, tmp_path, small_golden, small_golden_logs)
    assert max(res.history["dtime_s"]) == 150 * cfg.step_factor


def test_rejected_and_abort(tmp_path, small_golden_logs):
    cfg = small_config(n_steps=40, x_equilibrium=0.2)
    res = _run(cfg, three_precipitates(cfg), tmp_path)
    assert isinstance(res, kks_oracle.AdaptiveStepError)
    assert str(res) == small_golden_logs["rejected40"]["error"]
    for name in ("log.txt", "dtime.txt"):
        assert (tmp_path / name).read_text() == small_golden_logs["rejected40"][name]


def test_synthetic_microstructure_20_steps(tmp_path):
    from pf_kks_gpu import workloads

    g = np.load(os.path.join(GOLDEN, "reference_demo160.npz"))
    cfg, spec = workloads.demo160(n_steps=20)
    state = workloads.initial_state(cfg, spec)
    for name, a in zip(("eta", "X", "X_al", "X_th"), state):
        np.testing.assert_array_equal(a.ravel()[g[f"init_{name}_idx"]], g[f"init_{name}_val"])
    res = kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path))
    for name in FIELDS:
        flat = getattr(res, name).ravel()
        np.testing.assert_allclose(flat[g[f"final_{name}_idx"]], g[f"final_{name}_val"], rtol=0, atol=1e-12)
        assert flat.sum() == pytest.approx(float(g[f"final_{name}_sum"]), rel=1e-12)
    for name in HIST:
        np.testing.assert_allclose(np.asarray(res.history[name], float), g[f"h_{name}"], rtol=1e-9, atol=1e-14,
                                   equal_nan=True, err_msg=name)


def _reproducible_run_config(n_steps):
    """configs/reproducible_run.toml of the reference: the SimulationConfig defaults."""
    return SimulationConfig(n_steps=n_steps, material_tables=DEFAULT_TABLES)


def _archived_initial_state(cfg):
    ox, oy, oz, r = load_precipitates(DEFAULT_PRECIPITATES)
    return place_precipitates(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz, cfg.x_matrix, cfg.x_precipitate, r, ox,
                              oy, oz)


def test_first_step_matches_archived_map(tmp_path):
    """735^2 first step vs the map of the 2022 run (reference tests/test_archived_run.py:35-46, atol 1e-14)."""
    a = np.load(os.path.join(GOLDEN, "archived_735.npz"))
    cfg = _reproducible_run_config(1)
    res = kks_oracle.run(cfg, *_archived_initial_state(cfg), cfg.material_tables, out_dir=str(tmp_path))
    assert os.listdir(tmp_path / "saved_maps") == ["map0.07s_400_400.00K.npz"]
    with np.load(tmp_path / "saved_maps" / "map0.07s_400_400.00K.npz") as new:
        assert list(new.files) == list(a["map_files"])
        for name in FIELDS:
            flat = new[name].ravel()
            np.testing.assert_allclose(flat[a[f"map_{name}_idx"]], a[f"map_{name}_val"], rtol=0, atol=1e-14)
            assert flat.sum() == pytest.approx(float(a[f"map_{name}_sum"]), rel=1e-13)
            assert (flat * flat).sum() == pytest.approx(float(a[f"map_{name}_sumsq"]), rel=1e-13)
        for key in new.files:
            if key in FIELDS:
                continue
            ref = a[f"mapkey_{key}"]
            assert new[key].dtype == ref.dtype, key
            np.testing.assert_allclose(new[key], ref, rtol=0, atol=1e-14, err_msg=key)
    line = (tmp_path / "dtime.txt").read_text().splitlines()[1].rstrip()
    assert line == str(a["dtime_line1"])
    assert res.ttime == pytest.approx(float(a["mapkey_ttime"]), rel=1e-14)


def test_twenty_steps_match_archived_histories(tmp_path):
    """20 steps vs the archived histories (reference tests/test_archived_run.py:49-61, rtol 1e-12)."""
    a = np.load(os.path.join(GOLDEN, "archived_735.npz"))
    cfg = _reproducible_run_config(20)
    res = kks_oracle.run(cfg, *_archived_initial_state(cfg), cfg.material_tables, out_dir=str(tmp_path),
                         save_maps=False, write_logs=False)
    for ref_key, new_key in [("time_out", "time"), ("T_out", "T"), ("surf_out", "surf"),
                             ("X_al_mean_out", "X_al_mean"), ("X_th_mean_out", "X_th_mean"),
                             ("eta_mean_out", "eta_mean")]:
        np.testing.assert_allclose(np.asarray(res.history[new_key], float), a[f"hist20_{ref_key}"], rtol=1e-12,
                                   atol=0, err_msg=ref_key)


def test_logs_fixture_is_consistent():
    with open(os.path.join(GOLDEN, "reference_small_logs.json")) as f:
        logs = json.load(f)
    assert logs["rejected40"]["dtime.txt"].count("RE>resmax") == 49


@pytest.mark.parametrize("case", ["accepted30", "enlarged40"])
def test_resume_from_loop_state_is_exact(tmp_path, relaxed_state, small_golden, case):
    """The oracle restarted at a step boundary of an armed run from its
    complete loop state (fields, scalars, histories, the residual pair's last
    entry) continues exactly as the uninterrupted run: this is how device
    states are handed to the oracle at large step counts."""
    if case == "accepted30":
        cfg = small_config(n_steps=30, x_equilibrium=0.2)
    else:
        cfg = small_config(n_steps=40, x_equilibrium=0.2, dtime_s=60, dtime_max=150, residual_min=7.6e-4)
    full = kks_oracle.run(cfg, *copy_state(relaxed_state), cfg.material_tables, out_dir=str(tmp_path / "full"),
                          snapshot_steps={17})
    snap = full.snapshots[17]
    assert snap["flag"] == 1 and snap["good_step"] == 2
    part = kks_oracle.run(cfg, *copy_state(snap["state"]), cfg.material_tables, out_dir=str(tmp_path / "part"),
                          resume=snap)
    for name in FIELDS:
        np.testing.assert_array_equal(getattr(part, name), getattr(full, name), err_msg=name)
    for name in HIST:
        np.testing.assert_array_equal(np.asarray(part.history[name], float), np.asarray(full.history[name], float),
                                      err_msg=name)
    np.testing.assert_array_equal(full.X, small_golden[f"{case}_X"])
    full_log = (tmp_path / "full" / "log.txt").read_text().splitlines()
    part_log = (tmp_path / "part" / "log.txt").read_text().splitlines()
    assert part_log[1:] == full_log[-(len(part_log) - 1):]
