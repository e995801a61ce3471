"""The FP64 step's fused passes (csrc/kks_fft64.cu) against the FP64 step's
cuFFT passes and the oracle.

An FP64 cell runs the six shared-memory FFT passes of the mixed pipeline in
double precision by default (launch shape pipeline 1); pipeline 0 keeps the
cuFFT D2Z / Z2D transforms. Both compute the same FP64 step, so they agree to
the round-off of two FFT implementations: fields within 1e-12 relative L2 and
histories within rtol 1e-10 after a dozen steps, on grids that exercise every
stage kind (radices 2, 3, 4, 5, 7; the prime stages 11, 19 and 71; odd and
non-square sides), with the same adaptive decisions. The column tile only
regroups identical per-column work: every tile gives the same bits. The
reference's own parity cases (tests/test_gpu_parity.py) run through these
passes too, since they are the FP64 default.
"""

import numpy as np
import pytest

from conftest import copy_state, rel_l2, small_config, three_precipitates

pytestmark = pytest.mark.gpu


def _state(nx, ny, n_steps=12, seed=21):
    from pf_kks_gpu import workloads
    from pf_kks_gpu.generator import MicrostructureSpec

    cfg = workloads.base_config(nx=nx, ny=ny, n_steps=n_steps, n_map_saves=2, n_surface_samples=4)
    big = nx * ny > 10 ** 6
    spec = MicrostructureSpec(nx, ny, n_cells=40 if big else 3, n_particles=1200 if big else max(3, nx * ny // 600),
                              seed=seed)
    return cfg, workloads.initial_state(cfg, spec)


def _run(cfg, state, shape=None, steps=None, precision="fp64"):
    from pf_kks_gpu import solver
    from pf_kks_gpu.materials import MaterialTables

    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    c = solver.Cell(cfg, tables, precision=precision)
    try:
        if shape is not None:
            pipeline, cols = shape
            c.set_launch_shape(pipeline, cols, c.launch_shape()["field_blocks"])
        pipeline = c.launch_shape()["pipeline"]
        c.upload(*copy_state(state))
        st = c.run(cfg.n_steps if steps is None else steps)
        recs, rows = c.drain()
        return st, c.download(), rows, [(r.istep, r.kind) for r in recs], pipeline
    finally:
        c.close()


@pytest.mark.parametrize("shape", [(64, 64), (96, 80), (45, 38), (33, 64), (100, 80), (105, 98), (1420, 1420)])
def test_fused_fp64_matches_cufft_fp64(shape):
    nx, ny = shape
    cfg, state = _state(nx, ny, n_steps=4 if nx * ny > 10 ** 6 else 12)
    st_f, got, rows_f, dec_f, pipe_f = _run(cfg, state)
    assert pipe_f == 1, "the FP64 cell should default to the fused passes"
    st_c, ref, rows_c, dec_c, pipe_c = _run(cfg, state, shape=(0, 1))
    assert pipe_c == 0
    assert st_f == st_c == 0
    assert dec_f == dec_c
    for name, a, b in zip(("eta", "X", "X_al", "X_th"), got, ref):
        assert rel_l2(a, b) <= 1e-12, name
    np.testing.assert_allclose(rows_f, rows_c, rtol=1e-10, atol=1e-15)


def test_fused_fp64_column_tiles_give_the_same_bits():
    cfg, state = _state(96, 80)
    _, ref, ref_rows, _, _ = _run(cfg, state, shape=(1, 1))
    for cols in (2, 3, 4):
        _, got, rows, _, _ = _run(cfg, state, shape=(1, cols))
        for a, b in zip(got, ref):
            np.testing.assert_array_equal(a, b, err_msg=f"cols={cols}")
        np.testing.assert_allclose(rows, ref_rows, rtol=1e-12, atol=1e-15)


def test_fused_fp64_adaptive_decisions_match_cufft(relaxed_state):
    """Armed from step 1 (accepts and enlarges), and the rejection / abort case:
    the same decisions at the same steps as the cuFFT FP64 passes."""
    for cfg, state in ((small_config(n_steps=40, x_equilibrium=0.2, dtime_s=60, dtime_max=150, residual_min=7.6e-4),
                        relaxed_state),
                       (small_config(n_steps=40, x_equilibrium=0.2), None)):
        state = three_precipitates(cfg) if state is None else state
        st_f, got, rows_f, dec_f, _ = _run(cfg, state)
        st_c, ref, rows_c, dec_c, _ = _run(cfg, state, shape=(0, 1))
        assert st_f == st_c
        assert dec_f == dec_c and len(dec_f) > 0
        if st_f == 0:  # after a stop the buffers hold a rejected candidate: not a result
            for name, a, b in zip(("eta", "X"), got, ref):
                assert rel_l2(a, b) <= 1e-11, name
