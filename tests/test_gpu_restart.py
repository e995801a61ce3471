"""The oracle continued from a GPU state: the FP64 step's loop state at a step
boundary (fields, scalars, history rows and the residual pair's minus entry,
``kks_download_pair``) is handed to the oracle, which then runs the same steps
as the GPU. Both must take the same adaptive decisions at the same steps and
end in the same state (1e-10 relative L2) or stop at the same step with the
same error. This is how a long GPU run is checked against the oracle near its
end without running the oracle for the whole run (the 1420^2 record in
tests/accuracy/ramp1420_stop.py uses the same hand-over).
"""

import numpy as np
import pytest

from conftest import copy_state, rel_l2, small_config, three_precipitates

pytestmark = pytest.mark.gpu

FIELDS = ("eta", "X", "X_al", "X_th")


def _decisions_of_records(recs):
    from pf_kks_gpu import _lib as L

    kinds = {L.KKS_REC_REJECTED: "rejected", L.KKS_REC_ACCEPTED: "accepted", L.KKS_REC_ENLARGED: "enlarged"}
    return [(r.istep, kinds[r.kind]) for r in recs if r.kind in kinds]


def _decisions_of_oracle(attempts):
    return [(a["istep"], a["decision"]) for a in attempts if a["decision"] != "none"]


def test_oracle_continues_an_armed_gpu_run(tmp_path, relaxed_state):
    """The enlarged set-up of the reference's equivalence tests (accepted and
    enlarged steps): GPU steps 0..16, then the oracle from the GPU's state at
    step 17 against the GPU's own steps 17..39."""
    from conftest import gpu_loop_state
    from oracle import kks_oracle
    from pf_kks_gpu import solver
    from pf_kks_gpu.materials import MaterialTables

    cfg = small_config(n_steps=40, x_equilibrium=0.2, dtime_s=60, dtime_max=150, residual_min=7.6e-4)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    cell = solver.Cell(cfg, tables, precision="fp64")
    try:
        cell.upload(*relaxed_state)
        assert cell.run(17) == 0
        _, rows = cell.drain()
        resume, state = gpu_loop_state(cell, rows)
        assert resume["flag"] == 1 and resume["istep"] == 17
        assert cell.run(23) == 0
        recs, _ = cell.drain()
        gpu_final = cell.download()
    finally:
        cell.close()
    seen = []
    ref = kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path), resume=resume,
                         on_attempt=seen.append)
    assert _decisions_of_oracle(seen) == _decisions_of_records(recs)
    assert {d for _, d in _decisions_of_oracle(seen)} == {"accepted", "enlarged"}
    for name, a in zip(FIELDS, gpu_final):
        assert rel_l2(a, getattr(ref, name)) <= 1e-10, name


def test_oracle_stops_where_the_gpu_run_stops(tmp_path):
    """The rejection / abort set-up (three sharp precipitates, armed at step
    2): GPU steps 0..3, then the oracle from the GPU's state at step 4, where
    both reject until max_iterations and stop with the same error."""
    from conftest import gpu_loop_state
    from oracle import kks_oracle
    from pf_kks_gpu import _lib as L
    from pf_kks_gpu import solver
    from pf_kks_gpu.materials import MaterialTables

    cfg = small_config(n_steps=40, x_equilibrium=0.2)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    cell = solver.Cell(cfg, tables, precision="fp64")
    try:
        cell.upload(*three_precipitates(cfg))
        assert cell.run(4) == 0
        _, rows = cell.drain()
        resume, state = gpu_loop_state(cell, rows)
        assert cell.run(36) == L.KKS_STATUS_MAX_ITER
        recs, _ = cell.drain()
        s = cell.state()
    finally:
        cell.close()
    seen = []
    with pytest.raises(kks_oracle.AdaptiveStepError) as err:
        kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path), resume=resume,
                       on_attempt=seen.append)
    assert _decisions_of_oracle(seen) == _decisions_of_records(recs)
    assert str(err.value) == (f"step {s.error_istep}: no admissible time step after {s.error_iteration} attempts "
                              f"(dtime_s={s.error_dtime_s:.2e})")
