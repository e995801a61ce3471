"""Host-side logic of the drop-in (no GPU): configuration, schedule, maps,
logs, generator, history typing, ensemble partition."""

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, small_config

from pf_kks_gpu import config as C
from pf_kks_gpu import io as kio
from pf_kks_gpu import runlog, solver, workloads
from pf_kks_gpu.ensemble import cell_cost, partition
from pf_kks_gpu.generator import MicrostructureSpec, generate
from pf_kks_gpu.materials import DEFAULT_TABLES, MaterialTables


def test_config_defaults_are_the_reproducible_run():
    cfg = C.SimulationConfig()
    assert (cfg.nx, cfg.ny, cfg.nz, cfg.dx) == (735, 735, 1, 0.5e-9)
    assert (cfg.dtime_s, cfg.dtime_max, cfg.dtime_min_divisor) == (75, 400, 1000)
    assert (cfg.c_Meta, cfg.c_eps0, cfg.c_gamma, cfg.c_D) == (0.6, 0.25, 1, 1)
    assert (cfg.n_steps, cfg.n_map_saves, cfg.n_surface_samples) == (30000, 40, 500)
    assert cfg.lambd == 2.5 * cfg.dx and cfg.T_start == 400


def test_unknown_config_key_is_rejected(tmp_path):
    p = tmp_path / "bad.toml"
    p.write_text("[grid]\nnx = 10\nnot_a_key = 1\n")
    with pytest.raises(ValueError, match="not_a_key"):
        C.load_config(p)


def test_gpu_section_and_overrides(tmp_path):
    p = tmp_path / "c.toml"
    p.write_text("[grid]\nnx = 64\nny = 32\n[output]\nn_steps = 7\n[gpu]\nprecision = \"mixed\"\ndevice = 1\n")
    cfg = C.load_config(p, n_steps=9, fft_threads=None)
    assert (cfg.nx, cfg.ny, cfg.n_steps) == (64, 32, 9)
    assert cfg.gpu_options.precision == "mixed" and cfg.gpu_options.device == 1
    assert cfg.gpu_options.autotune is False
    assert "gpu" not in cfg.to_dict()
    p.write_text("[gpu]\nprecision = \"mixed\"\nautotune = true\n")
    assert C.load_config(p).gpu_options.autotune is True
    p.write_text("[gpu]\nprecision = \"fp16\"\n")
    with pytest.raises(ValueError):
        C.load_config(p)
    p.write_text("[gpu]\nbogus = 1\n")
    with pytest.raises(ValueError, match="bogus"):
        C.load_config(p)


def test_schedule_matches_reference_semantics():
    s = solver.Schedule.from_config(small_config(n_steps=40, n_map_saves=3, n_surface_samples=10))
    assert s.n_steps == 40 and s.map_steps == {1, 20, 40}
    assert 1 in s.surface_steps and 40 in s.surface_steps and len(s.surface_steps) == 10
    # a single map save makes a one-step run (pf_kks/solver.py:48-53)
    assert solver.Schedule.from_config(small_config(n_steps=40, n_map_saves=1)).n_steps == 1


def test_map_filename_roundtrip():
    name = kio.map_filename(2221.716369079099, 400, 722.5789845064727)
    assert name == "map2221.72s_400_722.58K"
    assert kio.parse_map_filename(name + ".npz") == (2221.72, 400.0, 722.58)


def test_runlog_matches_oracle_formats(tmp_path):
    from oracle import kks_oracle

    res = solver.Residual(-1.2345e-3, 7.06, -1.38e-1, 6.59e-8, 2.26e-11)
    a = runlog.RunLog(str(tmp_path / "a"))
    b = kks_oracle.RunLog(str(tmp_path / "b"))
    for log in (a, b):
        log.state(100, 402.4671, 2.8e-16, 5.22e-16, 1.78e-22, 1.02e-5, 75)
        log.rejected(4, 3, 0.06, res, 2580.0)
        log.accepted(5, res, 2580.0)
        log.enlarged(6, res, 2580.0)
    a.flush()
    for name in ("log.txt", "dtime.txt"):
        assert (tmp_path / "a" / name).read_text() == (tmp_path / "b" / name).read_text()


def test_history_builder_types():
    cfg = small_config(n_steps=3)
    hb = solver._HistoryBuilder(cfg, runlog.RunLog(".", enabled=False), False, 3)
    rows = np.zeros((3, 32))
    for k in range(3):
        rows[k, solver.L.H["istep"]] = k
        rows[k, solver.L.H["time_s"]] = 75.0 * (k + 1)
        rows[k, solver.L.H["dtime_s"]] = 75.0
        rows[k, solver.L.H["time"]] = 0.5 * k
    hb.rows(rows)
    assert hb.hist["time"][0] == 0 and isinstance(hb.hist["time"][0], int)
    assert all(isinstance(v, int) for v in hb.hist["time_s"])  # dtime_s = 75 (int) never changed
    assert np.asarray(hb.hist["time_s"]).dtype == np.int64


def test_generator_is_seeded_and_kks_consistent():
    t = MaterialTables.from_npz(DEFAULT_TABLES, 1.0, 0.25)
    coeffs = [t.at(400.0, n) for n in ("A_alp", "B_alp", "A_thet", "B_thet")]
    spec = MicrostructureSpec(96, 80, n_cells=4, n_particles=12, seed=5)
    a = generate(spec, *coeffs)
    b = generate(spec, *coeffs)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    c = generate(MicrostructureSpec(96, 80, n_cells=4, n_particles=12, seed=6), *coeffs)
    assert not np.array_equal(a[0], c[0])
    eta, X, X_al, X_th = a
    assert eta.shape == (96, 80, 1) and 0 <= eta.min() and eta.max() <= 1
    assert eta.max() > 0.99 and np.mean(eta < 0.05) > 0.5
    h = 3 * eta**2 - 2 * eta**3
    np.testing.assert_allclose((1 - h) * X_al + h * X_th, X, rtol=1e-12, atol=1e-14)
    matrix = X[eta < 1e-6]
    assert 0.048 <= matrix.min() and matrix.max() <= 0.052


def test_workloads_have_the_configured_sizes():
    cfg, spec = workloads.ramp1420(n_steps=100)
    assert (cfg.nx, cfg.ny) == (1420, 1420) and spec.n_particles == 1200 and spec.r_max == 10
    assert solver.Schedule.from_config(cfg).n_steps == 100
    assert cfg.schedule_temperature == [400.0, 719.0]
    assert cfg.schedule_time[1] == pytest.approx((719 - 400) * 3)
    ens = workloads.ensemble(n_instances=48, n_steps=10)
    assert len(ens) == 48 and {c.nx for c, _ in ens} <= set(workloads.ENSEMBLE_SIDES)
    from pf_kks_gpu.kinetics import quenched_vacancy_fraction

    assert quenched_vacancy_fraction(workloads.T_QUENCH_XV_1E4) == pytest.approx(1e-4, rel=1e-6)


def test_partition_balances_cost():
    sides = [128, 192, 256, 384, 512] * 4
    costs = [cell_cost(n, n, 100) for n in sides]
    shards = partition(costs, 4)
    assert sorted(i for s in shards for i in s) == list(range(len(sides)))
    loads = [sum(costs[i] for i in s) for s in shards]
    assert max(loads) / min(loads) < 1.1
    assert partition(costs, 4) == shards  # deterministic
    assert partition(costs, 1) == [list(range(len(sides)))]


def test_make_params_scaling():
    cfg = small_config(c_D=2.0, c_Meta=0.5, vacancy_sink_distance=100e-9)
    t = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    p = solver.make_params(cfg, t)
    assert p.D0 == pytest.approx(float(t.D0) * 2.0)
    assert p.Meta0 == pytest.approx(5.6e-8 * 0.5)
    assert p.Lv2 == pytest.approx(1e-14)
    assert p.surf_scale == pytest.approx(cfg.dx**2 / (2 * cfg.lambd))
    assert p.n_table == 6 and p.table_T[5] == 850.0


def test_golden_logs_present():
    with open(os.path.join(GOLDEN, "reference_small_logs.json")) as f:
        assert set(json.load(f)) == {"fixed40", "accepted30", "enlarged40", "rejected40"}


def test_accuracy_history_deviation_skips_shared_nans():
    from pf_kks_gpu.accuracy import history_deviation

    ref = np.array([1.0, 2.0, np.nan, 4.0])
    test = np.array([1.0, 2.5, np.nan, 4.0])
    d = history_deviation(test, ref)
    assert d["nan_mismatch"] == 0
    assert d["max_abs_dev"] == pytest.approx(0.5)
    assert d["max_dev_over_range"] == pytest.approx(0.5 / 3.0)
    d2 = history_deviation(np.array([1.0, np.nan, 3.0]), np.array([1.0, 2.0, 3.0]))
    assert d2["nan_mismatch"] == 1 and d2["max_abs_dev"] == 0.0
    assert "shape_test" in history_deviation(np.zeros(2), np.zeros(3))
