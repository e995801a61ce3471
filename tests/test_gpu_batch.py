"""Batched ensembles (``kks_batch_*``): the cells of a batch advance by one
launch per kernel for all of them, with each cell's dt, rejections, step
target and buffer parity on the device.

A batch run is deterministic: run twice it gives the same bits (fields, log
records, history rows). Against the same cells run alone (``kks_run``) it runs
the same stages on the same data in the same order, but in kernels compiled
separately, where the compiler may contract FP32 products differently; such a
difference in the FP32 increments of a mixed step is as large as the mixed
step's own rounding (1e-7 relative on X after a few dozen steps), so the bar
is the mixed path's: eta and X within 1e-6 relative L2, the FP32 phase
compositions within 1e-5, the same accept / enlarge / reject decisions, steps
and status, history rows within 1e-4 relative or 2e-7 absolute (the step
deltas of means of FP32-stored fields are round-off dominated). Covered: cells of different sizes, seeds
and schedules, step counts that differ per cell, adaptive cells that reject, a
cell that stops with MAX_ITER, single-cell runs between batch runs.
"""

import ctypes

import numpy as np
import pytest

from conftest import copy_state, rel_l2, small_config, three_precipitates

pytestmark = pytest.mark.gpu


def _members(relaxed):
    from pf_kks_gpu import workloads
    from pf_kks_gpu.generator import MicrostructureSpec

    out = []
    for k, (nx, ny, n) in enumerate([(128, 96, 30), (64, 64, 30), (96, 80, 30), (40, 50, 30)]):
        cfg = workloads.base_config(nx=nx, ny=ny, n_steps=n, n_map_saves=2, n_surface_samples=6)
        spec = MicrostructureSpec(nx, ny, n_cells=3, n_particles=max(3, nx * ny // 600), seed=20 + k)
        out.append((cfg, workloads.initial_state(cfg, spec)))
    # adaptive, armed from step 1 (accepts and enlarges; pf_kks tests' relaxed state)
    cfg = small_config(n_steps=40, x_equilibrium=0.2, dtime_s=60, dtime_max=150, residual_min=7.6e-4)
    out.append((cfg, relaxed))
    # adaptive from sharp precipitates: rejects until max_iterations (status MAX_ITER)
    cfg = small_config(n_steps=40, x_equilibrium=0.2)
    out.append((cfg, three_precipitates(cfg)))
    return out


def _cell(cfg, state, precision="mixed"):
    from pf_kks_gpu import solver
    from pf_kks_gpu.materials import MaterialTables

    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    c = solver.Cell(cfg, tables, precision=precision)
    c.upload(*copy_state(state))
    return c


def _alone(members, plan, precision="mixed"):
    """Each cell run alone through kks_run, in the given segments."""
    out = []
    for (cfg, state), segs in zip(members, plan):
        c = _cell(cfg, state, precision)
        recs, rows, st = [], [], 0
        for n in segs:
            st = c.run(n)
            r, w = c.drain()
            recs += r
            rows.append(w)
        out.append((c.download(), [bytes(r) for r in recs], np.concatenate(rows), st, c.state().istep))
        c.close()
    return out


def _batched(members, plan, single=None, groups=1):
    """All cells in one batch (split into ``groups`` streams), the same
    segments as kks_batch_run calls; ``single`` = (segment index, cell,
    steps): that cell also runs alone by kks_run after that segment (the batch
    must pick up its new parity)."""
    from pf_kks_gpu import _lib as L

    cells = [_cell(cfg, state) for cfg, state in members]
    lib = L.load()
    ptrs = (ctypes.c_void_p * len(cells))(*[c.h.value for c in cells])
    b = ctypes.c_void_p()
    L.check(lib.kks_batch_create(ptrs, len(cells), groups, ctypes.byref(b)), "kks_batch_create")
    recs = [[] for _ in cells]
    rows = [[] for _ in cells]
    status = [0] * len(cells)
    try:
        for s in range(max(len(p) for p in plan)):
            steps = (ctypes.c_int32 * len(cells))(*[p[s] if s < len(p) else 0 for p in plan])
            st = (ctypes.c_int32 * len(cells))()
            L.check(lib.kks_batch_run(b, steps, st), "kks_batch_run")
            for i, c in enumerate(cells):
                r, w = c.drain()
                recs[i] += [bytes(x) for x in r]
                rows[i].append(w)
                status[i] = st[i]
            if single is not None and single[0] == s:
                _, i, n = single
                status[i] = cells[i].run(n)
                r, w = cells[i].drain()
                recs[i] += [bytes(x) for x in r]
                rows[i].append(w)
        ms, att = ctypes.c_double(), ctypes.c_int64()
        L.check(lib.kks_batch_timing(b, ctypes.byref(ms), ctypes.byref(att)), "kks_batch_timing")
        assert att.value > 0 and ms.value > 0
        out = [(c.download(), recs[i], np.concatenate(rows[i]), status[i], c.state().istep)
               for i, c in enumerate(cells)]
    finally:
        L.check(lib.kks_batch_destroy(b), "kks_batch_destroy")
        for c in cells:
            c.close()
    return out


def _assert_fields_close(got, ref, what, tol=1e-6):
    for name, a, e in zip(("eta", "X", "X_al", "X_th"), got, ref):
        t = tol if name in ("eta", "X") else 10 * tol
        assert rel_l2(a, e) <= t, f"{what}: {name}"


def _assert_same(got, ref, field_tol=1e-6):
    """Batch against the cells alone: the mixed path's round-off, same decisions."""
    from pf_kks_gpu import _lib as L

    for i, (g, r) in enumerate(zip(got, ref)):
        _assert_fields_close(g[0], r[0], f"cell {i}", field_tol)
        assert len(g[1]) == len(r[1]), f"cell {i}: number of log records"
        for x, y in zip(g[1], r[1]):
            a, b = L.KksRecord.from_buffer_copy(x), L.KksRecord.from_buffer_copy(y)
            assert (a.kind, a.istep, a.iteration, a.good_step) == (b.kind, b.istep, b.iteration, b.good_step), \
                f"cell {i}: decisions differ"
            np.testing.assert_allclose([a.T, a.D, a.L, a.Meta, a.Vm, a.dtime_s],
                                       [b.T, b.D, b.L, b.Meta, b.Vm, b.dtime_s], rtol=1e-12)
        assert g[2].shape == r[2].shape, f"cell {i}: history rows"
        # the step deltas of means of FP32-stored fields (~1e-7) are round-off dominated
        np.testing.assert_allclose(g[2], r[2], rtol=1e-4, atol=2e-7, err_msg=f"cell {i}: history rows")
        assert g[3] == r[3], f"cell {i}: status"
        assert g[4] == r[4], f"cell {i}: step"


def _assert_identical(got, ref):
    """Two batch runs of the same inputs: bit for bit."""
    for i, (g, r) in enumerate(zip(got, ref)):
        for a, e in zip(g[0], r[0]):
            np.testing.assert_array_equal(a, e, err_msg=f"cell {i}")
        assert g[1] == r[1], f"cell {i}: log records"
        np.testing.assert_array_equal(g[2], r[2], err_msg=f"cell {i}: history rows")
        assert g[3:] == r[3:], f"cell {i}: status / step"


def test_batch_equals_cells_run_alone(relaxed_state):
    from pf_kks_gpu import _lib as L

    members = _members(relaxed_state)
    steps = [[30], [17], [25], [9], [40], [40]]
    ref = _alone(members, steps)
    got = _batched(members, steps)
    _assert_identical(_batched(members, steps), got)
    _assert_same(got, ref)
    # cost-balanced groups on their own streams: the same kernels per cell, the same bits
    _assert_identical(_batched(members, steps, groups=3), got)
    assert ref[-1][3] == L.KKS_STATUS_MAX_ITER  # the abort case stops on the device
    assert ref[-2][3] == L.KKS_STATUS_OK and ref[-2][4] == 40


def test_batch_segments_and_single_cell_runs_in_between(relaxed_state):
    """Several kks_batch_run calls, and a kks_run of one cell between two of
    them (odd step count: the cell's buffer parity changes outside the batch)."""
    members = _members(relaxed_state)[:5]
    plan = [[7, 11, 12], [5, 0, 12], [3, 4, 5], [9, 0, 0], [13, 14, 13]]
    # cell 1 runs 3 more steps alone after the first segment
    alone_plan = [[7, 11, 12], [5, 3, 0, 12], [3, 4, 5], [9, 0, 0], [13, 14, 13]]
    ref = _alone(members, alone_plan)
    got = _batched(members, plan, single=(0, 1, 3), groups=2)
    _assert_same(got, ref)


def test_batch_rejects_cells_it_cannot_share():
    from pf_kks_gpu import _lib as L
    from pf_kks_gpu import solver, workloads
    from pf_kks_gpu.materials import MaterialTables

    cfg = workloads.base_config(nx=64, ny=64, n_steps=4, n_map_saves=2, n_surface_samples=2)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    a = solver.Cell(cfg, tables, precision="mixed")
    f = solver.Cell(cfg, tables, precision="fp64")
    lib = L.load()
    b = ctypes.c_void_p()
    for cells in ([a, f], [a, a]):
        ptrs = (ctypes.c_void_p * 2)(*[c.h.value for c in cells])
        assert lib.kks_batch_create(ptrs, 2, 1, ctypes.byref(b)) != L.KKS_OK
    a.close()
    f.close()


def test_ensemble_runs_as_one_batch(relaxed_state):
    from pf_kks_gpu.ensemble import Ensemble

    ens = Ensemble(_members(relaxed_state)[:3], precision="mixed")
    try:
        assert ens.mode == "batch"
        assert ens.run([4, 2, 3]) == [0, 0, 0]
        assert [c.state().istep for c in ens.cells] == [4, 2, 3]
        assert ens.run_streams(2) == [0, 0, 0]
        assert [c.state().istep for c in ens.cells] == [6, 4, 5]
        assert ens.batch_timing()[1] == 4
    finally:
        ens.close()


def test_ensemble_tunes_the_batch(relaxed_state):
    """The batch's column tile is timed on the batch itself; the cells start
    from their initial state afterwards and run exactly as alone with the
    chosen shape."""
    from pf_kks_gpu.ensemble import Ensemble

    members = _members(relaxed_state)[:4]
    ens = Ensemble(members, precision="mixed", tune=True, tune_attempts=3)
    try:
        assert set(ens.batch_tile_ms) == {1, 2, 3, 4} and set(ens.mode_ms) == {"batch", "streams"}
        assert set(ens.batch_grid_ms) == {1, 4, 16}
        assert ens.mode == min(ens.mode_ms, key=ens.mode_ms.get)
        assert set(ens.batch_groups_ms) == {1, 2, 3, 4} and ens.groups in ens.batch_groups_ms
        tiles = {s["cols"] for s in ens.shapes.values()}
        assert len(tiles) == 1
        assert [c.state().istep for c in ens.cells] == [0, 0, 0, 0]
        assert ens.run(5) == [0, 0, 0, 0]
        got = [c.download() for c in ens.cells]
    finally:
        ens.close()
    for (cfg, state), g in zip(members, got):
        c = _cell(cfg, state)
        shape = ens.shapes[(cfg.nx, cfg.ny)]
        c.set_launch_shape(1, shape["cols"], shape["field_blocks"])
        c.run(5)
        _assert_fields_close(c.download(), g, f"{cfg.nx}x{cfg.ny}")
        c.close()


@pytest.mark.parametrize("shapes", [((40, 38), (60, 76), (45, 38)), ((1420, 1420), (1420, 1420))],
                         ids=["prime19", "prime71"])
def test_batch_with_a_prime_stage(shapes):
    """Batches whose cells share a large prime factor of the y axis (19, or 71
    as at 1420 = 4 * 5 * 71: the batched prime-stage kernels, ten-warp blocks)
    against the same cells run alone; odd and non-multiple-of-4 sides take the
    plain-load paths, 1420^2 the tensor copies."""
    from pf_kks_gpu import workloads
    from pf_kks_gpu.generator import MicrostructureSpec

    members = []
    for k, (nx, ny) in enumerate(shapes):
        cfg = workloads.base_config(nx=nx, ny=ny, n_steps=6, n_map_saves=2, n_surface_samples=3)
        big = nx * ny > 10 ** 6
        spec = MicrostructureSpec(nx, ny, n_cells=40 if big else 3, n_particles=1200 if big else 4, seed=30 + k)
        members.append((cfg, workloads.initial_state(cfg, spec)))
    plan = [[4]] * len(members)
    ref = _alone(members, plan)
    got = _batched(members, plan, groups=2)
    _assert_same(got, ref)
    # and both within the mixed step's bar of the FP64 step
    f64 = _alone(members, plan, precision="fp64")
    for i, (g, e) in enumerate(zip(got, f64)):
        for k, name in enumerate(("eta", "X")):
            assert rel_l2(g[0][k], e[0][k]) <= 1e-6, f"cell {i} batch vs fp64: {name}"


def test_concurrent_prime71_cells_finish():
    """Two 1420^2 cells advanced concurrently, as two stream groups of a batch
    and on their own streams (kks_run_many), three times each: every run
    reaches its target with status OK and the same bits as the cells alone.
    (The column passes once re-armed their copy barrier for a second copy
    before every thread had seen the first complete; a warp delayed by the
    other cell's blocks then waited on a phase that could not complete, the
    bounded wait ran out, and the run stopped with KKS_STATUS_TIMEOUT. And the
    first column pass once rewrote its FT(eta) columns in place while a
    delayed warp was still copying them out: one spectral mode of the kept
    FT(eta) came out wrong now and then, and the fields drifted by 1e-10.)"""
    from pf_kks_gpu import _lib as L
    from pf_kks_gpu import workloads
    from pf_kks_gpu.generator import MicrostructureSpec

    members = []
    for k in range(2):
        cfg = workloads.base_config(nx=1420, ny=1420, n_steps=6, n_map_saves=2, n_surface_samples=3)
        spec = MicrostructureSpec(1420, 1420, n_cells=40, n_particles=1200, seed=30 + k)
        members.append((cfg, workloads.initial_state(cfg, spec)))
    plan = [[4]] * 2
    ref = _alone(members, plan)
    for _ in range(3):
        got = _batched(members, plan, groups=2)
        for i, (g, r) in enumerate(zip(got, ref)):
            assert g[3] == L.KKS_STATUS_OK and g[4] == 4, f"batch cell {i}: status {g[3]}, step {g[4]}"
            for a, b in zip(g[0], r[0]):
                np.testing.assert_array_equal(a, b)
    cells = [_cell(cfg, st) for cfg, st in members]
    try:
        ptrs = (ctypes.c_void_p * 2)(*[c.h.value for c in cells])
        for _ in range(3):
            for c, (cfg, st) in zip(cells, members):
                c.upload(*copy_state(st))
            steps = (ctypes.c_int32 * 2)(4, 4)
            status = (ctypes.c_int32 * 2)()
            L.check(L.load().kks_run_many(ptrs, 2, steps, status), "kks_run_many")
            for i, c in enumerate(cells):
                assert status[i] == L.KKS_STATUS_OK and c.state().istep == 4, f"cell {i}: status {status[i]}"
                for a, b in zip(c.download(), ref[i][0]):
                    np.testing.assert_array_equal(a, b)
    finally:
        for c in cells:
            c.close()
