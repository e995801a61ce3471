"""Launch shapes and the autotuner (``kks_get/set_launch_shape``,
``kks_autotune``, ``pf_kks_gpu.autotune``).

A launch shape only changes how the work of an attempt is cut into blocks: in
unarmed steps (fixed dt, no residual decision) every shape of the fused passes
gives the same fields bit for bit, and the cuFFT passes agree to FP32
round-off. The autotuner leaves the cell's state, step and records as it found
them, and a batch takes every cell with its own shape (its results match the
cells run alone to the mixed path's round-off).
"""

import ctypes

import numpy as np
import pytest

from conftest import copy_state, rel_l2

pytestmark = pytest.mark.gpu


def _member(nx, ny, n_steps=24, seed=5):
    from pf_kks_gpu import workloads
    from pf_kks_gpu.generator import MicrostructureSpec

    cfg = workloads.base_config(nx=nx, ny=ny, n_steps=n_steps, n_map_saves=2, n_surface_samples=4)
    spec = MicrostructureSpec(nx, ny, n_cells=3, n_particles=max(3, nx * ny // 600), seed=seed)
    return cfg, workloads.initial_state(cfg, spec)


def _cell(cfg, state, precision="mixed"):
    from pf_kks_gpu import solver
    from pf_kks_gpu.materials import MaterialTables

    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    c = solver.Cell(cfg, tables, precision=precision)
    c.upload(*copy_state(state))
    return c


def _run(cell, n):
    st = cell.run(n)
    _, rows = cell.drain()
    return st, cell.download(), rows


def test_shapes_give_the_same_fields():
    cfg, state = _member(96, 80)
    ref_cell = _cell(cfg, state)
    default = ref_cell.launch_shape()
    assert default["pipeline"] == 1 and default["cols"] == 3
    cap = default["field_blocks"]
    st, ref, ref_rows = _run(ref_cell, 8)
    ref_cell.close()
    assert st == 0
    for cols, fb in ((1, 1), (2, max(1, cap // 3)), (4, cap)):
        c = _cell(cfg, state)
        c.set_launch_shape(1, cols, fb)
        assert c.launch_shape() == {"pipeline": 1, "cols": cols, "field_blocks": fb}
        st, got, rows = _run(c, 8)
        c.close()
        assert st == 0
        for a, b in zip(got, ref):
            np.testing.assert_array_equal(a, b, err_msg=f"cols={cols} field_blocks={fb}")
        np.testing.assert_allclose(rows, ref_rows, rtol=1e-11, atol=1e-14)
    c = _cell(cfg, state)
    c.set_launch_shape(0, 3, cap)  # the cuFFT passes
    st, got, _ = _run(c, 8)
    c.close()
    for name, a, b in zip(("eta", "X"), got[:2], ref[:2]):
        assert rel_l2(a, b) <= 1e-6, name


def test_invalid_shapes_are_rejected():
    from pf_kks_gpu import _lib as L

    cfg, state = _member(64, 64)
    c = _cell(cfg, state)
    f = _cell(cfg, state, precision="fp64")
    try:
        for args in ((1, 5, 8), (1, 0, 8), (1, 3, 0), (1, 3, 10 ** 6), (2, 3, 8)):
            with pytest.raises(L.KksError):
                c.set_launch_shape(*args)
        with pytest.raises(L.KksError):
            f.set_launch_shape(1, 5, 8)  # the FP64 passes take the same column tiles
        f.set_launch_shape(1, 2, 8)
        assert f.launch_shape() == {"pipeline": 1, "cols": 2, "field_blocks": 8}
        f.set_launch_shape(0, 2, 4)
        assert f.launch_shape()["field_blocks"] == 4 and f.launch_shape()["pipeline"] == 0
    finally:
        c.close()
        f.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_autotune_restores_the_state(precision):
    cfg, state = _member(128, 96)
    a = _cell(cfg, state, precision)
    a.run(3)
    a.drain()
    before = a.download()
    s0 = a.state()
    shape, ms = a.autotune(attempts=6)
    assert ms > 0
    s1 = a.state()
    assert (s1.istep, s1.n_records, s1.n_rows, s1.parity) == (s0.istep, s0.n_records, s0.n_rows, s0.parity)
    for x, y in zip(a.download(), before):
        np.testing.assert_array_equal(x, y)
    recs, rows = a.drain()
    assert len(recs) == 0 and len(rows) == 0
    assert a.launch_shape() == shape
    # the run goes on from the same state as an untuned cell
    b = _cell(cfg, state, precision)
    b.run(3)
    b.drain()
    _, ra, _ = _run(a, 6)
    _, rb, _ = _run(b, 6)
    a.close()
    b.close()
    for name, x, y in zip(("eta", "X"), ra[:2], rb[:2]):
        assert rel_l2(x, y) <= (1e-6 if precision == "mixed" else 1e-12), name


def test_autotune_cache(tmp_path, monkeypatch):
    from pf_kks_gpu import autotune

    monkeypatch.setenv("KKS_AUTOTUNE_CACHE", str(tmp_path / "shapes.json"))
    cfg, state = _member(64, 64)
    a = _cell(cfg, state)
    r1 = autotune.tune(a, attempts=4)
    b = _cell(cfg, state)
    r2 = autotune.tune(b, attempts=4)
    assert r1["source"] == "measured" and r2["source"] == "cache"
    assert r2["shape"] == r1["shape"] == b.launch_shape()
    c = _cell(cfg, state)
    r3 = autotune.tune(c, attempts=4, batchable=True)
    assert r3["shape"]["pipeline"] == 1
    for x in (a, b, c):
        x.close()


def test_batch_takes_each_cells_shape():
    from pf_kks_gpu import _lib as L

    members = [_member(96, 80, seed=1), _member(64, 64, seed=2), _member(128, 96, seed=3)]
    shapes = [(1, 2, 7), (1, 4, 16), (1, 1, 48)]
    ref = []
    for (cfg, state), sh in zip(members, shapes):
        c = _cell(cfg, state)
        c.set_launch_shape(*sh)
        ref.append(_run(c, 9)[1])
        c.close()
    cells = []
    for (cfg, state), sh in zip(members, shapes):
        c = _cell(cfg, state)
        c.set_launch_shape(*sh)
        cells.append(c)
    lib = L.load()
    ptrs = (ctypes.c_void_p * 3)(*[c.h.value for c in cells])
    b = ctypes.c_void_p()
    L.check(lib.kks_batch_create(ptrs, 3, 1, ctypes.byref(b)), "kks_batch_create")
    try:
        with pytest.raises(L.KksError):
            cells[0].set_launch_shape(1, 3, 7)  # fixed while the cell is in a batch
        steps = (ctypes.c_int32 * 3)(9, 9, 9)
        st = (ctypes.c_int32 * 3)()
        L.check(lib.kks_batch_run(b, steps, st), "kks_batch_run")
        assert list(st) == [0, 0, 0]
        for c, r in zip(cells, ref):
            for name, x, y in zip(("eta", "X", "X_al", "X_th"), c.download(), r):
                # batched kernels: the single-cell run to the mixed path's round-off
                assert rel_l2(x, y) <= (1e-6 if name in ("eta", "X") else 1e-5), name
    finally:
        L.check(lib.kks_batch_destroy(b), "kks_batch_destroy")
        cells[0].set_launch_shape(1, 3, 7)  # free again once the batch is gone
        for c in cells:
            c.close()


def test_solver_run_with_autotune(tmp_path, monkeypatch):
    """``[gpu] autotune = true``: solver.run tunes the cell on its initial
    state (cached), and the run itself is the untuned run to the mixed bar."""
    from pf_kks_gpu import solver

    monkeypatch.setenv("KKS_AUTOTUNE_CACHE", str(tmp_path / "shapes.json"))
    cfg, state = _member(96, 80, n_steps=12)
    ref = solver.run(cfg, *copy_state(state), out_dir=str(tmp_path / "plain"), verbose=False, precision="mixed")
    opts = cfg.gpu_options
    opts.autotune = True
    cfg.gpu = opts
    got = solver.run(cfg, *copy_state(state), out_dir=str(tmp_path / "tuned"), verbose=False, precision="mixed")
    for name in ("eta", "X"):
        assert rel_l2(getattr(got, name), getattr(ref, name)) <= 1e-6, name
    assert len(got.history["time"]) == len(ref.history["time"])
    assert (tmp_path / "shapes.json").exists()
