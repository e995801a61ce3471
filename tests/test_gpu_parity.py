"""Parity of the CUDA step with the oracle and with the reference's own outputs.

FP64 path: fields within 1e-10 relative L2 (the bar of the plain GPU step),
histories within rtol 1e-9, the same accept / enlarge / reject sequence and
byte-identical log files, on the set-ups of the reference's equivalence tests
(tests/test_solver_equivalence.py:79-118 of the reference) and on the
synthetic 160^2 microstructure.

Mixed path (FP32 transforms and pointwise math on the step increments, FP64
state): within 1e-6 relative L2 of the FP64 oracle on eta and X, mass (the
mean of X) conserved to FP64 round-off.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN, assert_logs_equivalent, copy_state, rel_l2, small_config, three_precipitates

pytestmark = pytest.mark.gpu

FIELDS = ("X", "X_al", "X_th", "eta")
HIST = ("eta_mean", "deta_mean", "X_mean", "X_al_mean", "dX_al_mean", "X_th_mean", "dX_th_mean", "dT", "T",
        "dtime", "time", "time_s", "surf", "dsurf", "L", "energy_s", "dtime_s", "residual_total",
        "residual_energy_derivative", "residual_diffusion", "residual_allen_cahn", "residual_temperature")
FIELD_TOL = 1e-10


def _run_gpu(cfg, state, out_dir, precision="fp64"):
    from pf_kks_gpu import solver

    try:
        return solver.run(cfg, *copy_state(state), out_dir=str(out_dir), verbose=False, precision=precision)
    except solver.AdaptiveStepError as exc:
        return exc


def _assert_hist_close(new_hist, ref_get, rtol=1e-9, atol=1e-13):
    for name in HIST:
        a = np.asarray(new_hist[name], dtype=np.float64)
        b = np.asarray(ref_get(name), dtype=np.float64)
        assert a.shape == b.shape, name
        np.testing.assert_allclose(a, b, rtol=rtol, atol=atol, equal_nan=True, err_msg=name)


def _assert_logs(out_dir, logs, exact=True):
    for name in ("log.txt", "dtime.txt"):
        with open(os.path.join(out_dir, name)) as f:
            text = f.read()
        if exact:
            assert text == logs[name], name
        else:
            assert_logs_equivalent(text, logs[name])
    assert sorted(os.listdir(os.path.join(out_dir, "saved_maps"))) == logs["maps"]


def test_fixed_steps_match_reference(tmp_path, small_golden, small_golden_logs):
    cfg = small_config(n_steps=40)
    res = _run_gpu(cfg, three_precipitates(cfg), tmp_path)
    g = small_golden
    for name in FIELDS:
        assert rel_l2(getattr(res, name), g[f"fixed40_{name}"]) <= FIELD_TOL, name
    _assert_hist_close(res.history, lambda n: g[f"fixed40_h_{n}"])
    assert res.good_step is None
    assert res.ttime == pytest.approx(float(g["fixed40_ttime"]), rel=1e-14)
    _assert_logs(tmp_path, small_golden_logs["fixed40"])
    assert rel_l2(res.sig_el, g["fixed40_sig_el"]) <= FIELD_TOL
    assert rel_l2(res.eps_el, g["fixed40_eps_el"]) <= FIELD_TOL


def test_accepted_adaptive_steps(tmp_path, relaxed_state, small_golden, small_golden_logs):
    cfg = small_config(n_steps=30, x_equilibrium=0.2)
    res = _run_gpu(cfg, relaxed_state, tmp_path)
    g = small_golden
    for name in FIELDS:
        assert rel_l2(getattr(res, name), g[f"accepted30_{name}"]) <= FIELD_TOL, name
    _assert_hist_close(res.history, lambda n: g[f"accepted30_h_{n}"], rtol=1e-8, atol=1e-12)
    assert res.good_step == 2
    _assert_logs(tmp_path, small_golden_logs["accepted30"])
    assert "We get  (resmin <RE <resmax)" in (tmp_path / "log.txt").read_text()


def test_enlarged_adaptive_steps(tmp_path, relaxed_state, small_golden, small_golden_logs):
    cfg = small_config(n_steps=40, x_equilibrium=0.2, dtime_s=60, dtime_max=150, residual_min=7.6e-4)
    res = _run_gpu(cfg, relaxed_state, tmp_path)
    g = small_golden
    for name in FIELDS:
        assert rel_l2(getattr(res, name), g[f"enlarged40_{name}"]) <= FIELD_TOL, name
    _assert_hist_close(res.history, lambda n: g[f"enlarged40_h_{n}"], rtol=1e-8, atol=1e-12)
    log = (tmp_path / "log.txt").read_text()
    assert "RE <resmin" in log and "We get  (resmin <RE <resmax)" in log
    assert max(res.history["dtime_s"]) == 150 * cfg.step_factor
    _assert_logs(tmp_path, small_golden_logs["enlarged40"])


def test_rejected_steps_and_abort(tmp_path, small_golden_logs):
    from pf_kks_gpu import solver

    cfg = small_config(n_steps=40, x_equilibrium=0.2)
    res = _run_gpu(cfg, three_precipitates(cfg), tmp_path)
    assert isinstance(res, solver.AdaptiveStepError)
    assert str(res) == small_golden_logs["rejected40"]["error"]
    assert (tmp_path / "dtime.txt").read_text().count("RE>resmax") == cfg.max_iterations - 1
    # From the unrelaxed state the step shrinks to dtime_s / 1000 and the
    # temperature term (a sum of G+ - G- over nearly equal states) is pure
    # round-off; its printed third digit depends on the FFT library's rounding.
    # Same lines, decisions and integers; reals within one unit of the printed
    # last digit.
    _assert_logs(tmp_path, small_golden_logs["rejected40"], exact=False)


def test_against_oracle_on_synthetic_microstructure(tmp_path):
    from oracle import kks_oracle
    from pf_kks_gpu import workloads

    cfg, spec = workloads.demo160(n_steps=20)
    state = workloads.initial_state(cfg, spec)
    res = _run_gpu(cfg, state, tmp_path / "gpu")
    ref = kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path / "cpu"))
    for name in FIELDS:
        assert rel_l2(getattr(res, name), getattr(ref, name)) <= FIELD_TOL, name
    _assert_hist_close(res.history, lambda n: ref.history[n])
    g = np.load(os.path.join(GOLDEN, "reference_demo160.npz"))
    for name in FIELDS:
        flat = getattr(res, name).ravel()
        np.testing.assert_allclose(flat[g[f"final_{name}_idx"]], g[f"final_{name}_val"], rtol=0, atol=1e-11)


@pytest.mark.parametrize("shape", [(45, 38), (33, 64), (64, 31)])
def test_odd_and_rectangular_grids(tmp_path, shape):
    from oracle import kks_oracle
    from pf_kks_gpu import workloads
    from pf_kks_gpu.generator import MicrostructureSpec

    nx, ny = shape
    cfg = workloads.base_config(nx=nx, ny=ny, n_steps=12, n_map_saves=2, n_surface_samples=5)
    spec = MicrostructureSpec(nx, ny, n_cells=3, n_particles=6, seed=3)
    state = workloads.initial_state(cfg, spec)
    res = _run_gpu(cfg, state, tmp_path / "gpu")
    ref = kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path / "cpu"))
    for name in FIELDS:
        assert rel_l2(getattr(res, name), getattr(ref, name)) <= FIELD_TOL, name
    _assert_hist_close(res.history, lambda n: ref.history[n])
    for log in ("log.txt", "dtime.txt"):
        assert (tmp_path / "gpu" / log).read_text() == (tmp_path / "cpu" / log).read_text()


def test_mixed_precision_close_to_fp64(tmp_path):
    from oracle import kks_oracle
    from pf_kks_gpu import workloads

    cfg, spec = workloads.demo160(n_steps=20)
    state = workloads.initial_state(cfg, spec)
    res = _run_gpu(cfg, state, tmp_path / "gpu", precision="mixed")
    ref = kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path / "cpu"))
    for name in ("eta", "X"):
        assert rel_l2(getattr(res, name), getattr(ref, name)) <= 1e-6, name
    # The FP32 transforms carry only the increment of X, whose mean mode is
    # exactly zero: the mass drifts only by the FP32 round-off of the
    # increments (~1e-12 per step here), not of the field.
    assert abs(res.X.mean() - state[1].mean()) <= 1e-10
    assert res.history["X_al_mean"][-1] == pytest.approx(ref.history["X_al_mean"][-1], rel=1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_checkpoint_restore_is_exact(precision):
    from pf_kks_gpu import solver, workloads
    from pf_kks_gpu.materials import MaterialTables

    cfg, spec = workloads.demo160(n_steps=40, precision=precision)
    cfg.x_equilibrium = 0.2  # arm the adaptive scheme early: the residual pair is part of the restart state
    state = workloads.initial_state(cfg, spec)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    a = solver.Cell(cfg, tables, precision=precision)
    a.upload(*state)
    a.run(10)
    blob = a.checkpoint()
    a.run(15)
    ref = a.download()
    b = solver.Cell(cfg, tables, precision=precision)
    b.restore(blob)
    b.run(15)
    got = b.download()
    for x, y in zip(got, ref):
        np.testing.assert_array_equal(x, y)
    assert b.state().istep == a.state().istep == 25
    a.close()
    b.close()


@pytest.mark.parametrize("shape", [(160, 160), (45, 38), (33, 64), (64, 31), (40, 50), (100, 80), (128, 192),
                                   (384, 96), (256, 512)])
def test_fused_fft_path_matches_oracle(tmp_path, shape):
    """The mixed step with the hand-written shared-memory FFTs (radices 2, 3,
    4, 5, 7 and the prime stages 11, 19, 71) against the FP64 oracle, and
    against the same step with cuFFT transforms. (64 x 31 has a prime factor
    without a direct stage and runs cuFFT; 128 x 192, 384 x 96 and 256 x 512
    are sides of the ensemble workload.)"""
    from oracle import kks_oracle
    from pf_kks_gpu import workloads
    from pf_kks_gpu.generator import MicrostructureSpec

    nx, ny = shape
    cfg = workloads.base_config(nx=nx, ny=ny, n_steps=15, n_map_saves=2, n_surface_samples=5)
    spec = MicrostructureSpec(nx, ny, n_cells=3, n_particles=max(3, nx * ny // 600), seed=11)
    state = workloads.initial_state(cfg, spec)
    fused = _run_gpu(cfg, state, tmp_path / "fused", precision="mixed")
    cuf = _run_gpu(cfg, state, tmp_path / "cufft", precision="mixed-cufft")
    ref = kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path / "cpu"))
    for name in ("eta", "X"):
        assert rel_l2(getattr(fused, name), getattr(ref, name)) <= 1e-6, name
        assert rel_l2(getattr(fused, name), getattr(cuf, name)) <= 1e-6, name
    for name in ("X_al", "X_th"):
        assert rel_l2(getattr(fused, name), getattr(ref, name)) <= 1e-5, name
    for name in ("eta_mean", "X_al_mean", "surf", "energy_s"):
        np.testing.assert_allclose(np.asarray(fused.history[name], float), np.asarray(ref.history[name], float),
                                   rtol=1e-5, atol=1e-12, err_msg=name)
    # mass moves only by the FP32 round-off of the increments (large on these
    # small, sharp initial states)
    assert abs(fused.X.mean() - state[1].mean()) <= 1e-8


def test_fused_fft_1420_short_run(tmp_path):
    """The bench grid (1420 = 4 * 5 * 71): three steps of the FP64 step and of
    the fused mixed step against the oracle."""
    from oracle import kks_oracle
    from pf_kks_gpu import workloads

    cfg, spec = workloads.ramp1420(n_steps=3)
    state = workloads.initial_state(cfg, spec)
    fused = _run_gpu(cfg, state, tmp_path / "fused", precision="mixed")
    assert fused.__class__.__name__ == "SimulationResult", fused
    f64 = _run_gpu(cfg, state, tmp_path / "fp64", precision="fp64")
    ref = kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path / "cpu"),
                         fft_workers=os.cpu_count())
    for name in FIELDS:
        assert rel_l2(getattr(f64, name), getattr(ref, name)) <= FIELD_TOL, name
    _assert_hist_close(f64.history, lambda n: ref.history[n])
    for name in ("eta", "X"):
        assert rel_l2(getattr(fused, name), getattr(ref, name)) <= 1e-6, name
    np.testing.assert_allclose(fused.history["energy_s"], ref.history["energy_s"], rtol=1e-6)


# ---------------------------------------------------------------------------
# Parity at the grids the benchmark configurations are quoted on.


def _archived_735(n_steps):
    """The reproducible run of the reference (configs/reproducible_run.toml:
    the SimulationConfig defaults, 735^2) from the archived precipitates."""
    from pf_kks_gpu.config import SimulationConfig
    from pf_kks_gpu.materials import DEFAULT_PRECIPITATES, DEFAULT_TABLES
    from pf_kks_gpu.microstructure import load_precipitates, place_precipitates

    cfg = SimulationConfig(n_steps=n_steps, material_tables=DEFAULT_TABLES)
    ox, oy, oz, r = load_precipitates(DEFAULT_PRECIPITATES)
    state = place_precipitates(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz, cfg.x_matrix, cfg.x_precipitate, r,
                               ox, oy, oz)
    return cfg, state


def test_fp64_first_step_matches_archived_map(tmp_path):
    """The FP64 GPU step against the map the reference's 2022 run archived
    after its first step (reference tests/test_archived_run.py:35-46): the map
    name and keys, every field at the sampled points within atol 1e-14 (the
    reference's own bar), the field sums, the history keys and the first
    dtime.txt line."""
    a = np.load(os.path.join(GOLDEN, "archived_735.npz"))
    cfg, state = _archived_735(1)
    res = _run_gpu(cfg, state, tmp_path)
    assert os.listdir(tmp_path / "saved_maps") == ["map0.07s_400_400.00K.npz"]
    with np.load(tmp_path / "saved_maps" / "map0.07s_400_400.00K.npz") as new:
        assert list(new.files) == list(a["map_files"])
        for name in FIELDS:
            flat = new[name].ravel()
            np.testing.assert_allclose(flat[a[f"map_{name}_idx"]], a[f"map_{name}_val"], rtol=0, atol=1e-14,
                                       err_msg=name)
            assert flat.sum() == pytest.approx(float(a[f"map_{name}_sum"]), rel=1e-13)
            assert (flat * flat).sum() == pytest.approx(float(a[f"map_{name}_sumsq"]), rel=1e-13)
        for key in new.files:
            if key not in FIELDS:
                assert new[key].dtype == a[f"mapkey_{key}"].dtype, key
                np.testing.assert_allclose(new[key], a[f"mapkey_{key}"], rtol=0, atol=1e-14, err_msg=key)
    line = (tmp_path / "dtime.txt").read_text().splitlines()[1].rstrip()
    assert line == str(a["dtime_line1"])
    assert res.ttime == pytest.approx(float(a["mapkey_ttime"]), rel=1e-14)


def test_fp64_twenty_steps_match_archived_histories(tmp_path):
    """20 FP64 GPU steps against the archived histories of the 2022 run
    (reference tests/test_archived_run.py:49-61, rtol 1e-12)."""
    a = np.load(os.path.join(GOLDEN, "archived_735.npz"))
    cfg, state = _archived_735(20)
    res = _run_gpu(cfg, state, tmp_path)
    for ref_key, new_key in [("time_out", "time"), ("T_out", "T"), ("surf_out", "surf"),
                             ("X_al_mean_out", "X_al_mean"), ("X_th_mean_out", "X_th_mean"),
                             ("eta_mean_out", "eta_mean")]:
        np.testing.assert_allclose(np.asarray(res.history[new_key], float), a[f"hist20_{ref_key}"], rtol=1e-12,
                                   atol=0, err_msg=ref_key)


def _assert_config2_scalars(res, ref, rtol):
    """The history scalars the 735^2 precision check reports: matrix Si mean,
    precipitate fraction (mean eta) and interface measure, every step."""
    for name in ("X_al_mean", "eta_mean", "surf"):
        np.testing.assert_allclose(np.asarray(res.history[name], float), np.asarray(ref.history[name], float),
                                   rtol=rtol, atol=1e-15, err_msg=name)


def test_iso735_fp64_and_mixed_against_oracle(tmp_path):
    """The 735^2 precision check (735 = 3 * 5 * 7^2: the fused passes with
    radices 3, 5, 7), isothermal 500 K, fixed dt, 30 steps: the FP64 step
    within 1e-10 relative L2 of the oracle on every field and 1e-9 on every
    history; the mixed step within 1e-6 on eta and X and on the matrix Si
    mean, precipitate fraction and interface measure."""
    from oracle import kks_oracle
    from pf_kks_gpu import solver, workloads

    cfg, spec = workloads.iso735(n_steps=30)
    state = workloads.initial_state(cfg, spec)
    ref = kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path / "cpu"),
                         fft_workers=os.cpu_count())
    f64 = _run_gpu(cfg, state, tmp_path / "fp64", precision="fp64")
    for name in FIELDS:
        assert rel_l2(getattr(f64, name), getattr(ref, name)) <= FIELD_TOL, name
    _assert_hist_close(f64.history, lambda n: ref.history[n])
    cell = solver.Cell(cfg, solver.MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0),
                       precision="mixed")
    assert cell.pipeline()[0], "735^2 should run the fused passes"
    cell.close()
    mixed = _run_gpu(cfg, state, tmp_path / "mixed", precision="mixed")
    for name in ("eta", "X"):
        assert rel_l2(getattr(mixed, name), getattr(ref, name)) <= 1e-6, name
    _assert_config2_scalars(mixed, ref, rtol=1e-6)
    assert abs(mixed.X.mean() - state[1].mean()) <= 1e-9


def _decisions(log_text):
    """(step, kind) of every adaptive decision in a log.txt."""
    out = []
    for line in log_text.splitlines():
        if ": RE>resmax" in line:
            out.append((int(line.split()[1].rstrip(":")), "rejected"))
        elif "(resmin <RE <resmax)" in line:
            out.append((int(line.split()[1].rstrip(",")), "accepted"))
        elif ":RE <resmin" in line:
            out.append((int(line.split()[-1]), "enlarged"))
    return out


@pytest.mark.parametrize("case", ["accepted30", "enlarged40"])
def test_mixed_decisions_match_reference(tmp_path, relaxed_state, small_golden, small_golden_logs, case):
    """The mixed step on the reference's accepted and enlarged set-ups
    (reference tests/test_solver_equivalence.py:89-107): the same adaptive
    decisions at the same steps as pf_kks, the same good_step, and fields
    within the mixed path's 1e-6 of the reference's."""
    from pf_kks_gpu import solver

    if case == "accepted30":
        cfg = small_config(n_steps=30, x_equilibrium=0.2)
    else:
        cfg = small_config(n_steps=40, x_equilibrium=0.2, dtime_s=60, dtime_max=150, residual_min=7.6e-4)
    res = _run_gpu(cfg, relaxed_state, tmp_path, precision="mixed")
    assert isinstance(res, solver.SimulationResult), res
    ref_decisions = _decisions(small_golden_logs[case]["log.txt"])
    assert ref_decisions, case
    assert _decisions((tmp_path / "log.txt").read_text()) == ref_decisions
    g = small_golden
    assert res.good_step == int(g[f"{case}_good_step"])
    np.testing.assert_array_equal(res.history["dtime_s"], g[f"{case}_h_dtime_s"])
    for name in ("eta", "X"):
        assert rel_l2(getattr(res, name), g[f"{case}_{name}"]) <= 1e-6, name
