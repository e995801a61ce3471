"""Failure detection on the GPU without a GPU fault.

The fused passes of the mixed path wait for their bulk / tensor copies on an
mbarrier with a bounded number of polls. Here the first wait of every pass is
given no polls at all (kks_set_wait_polls(0)): the wait runs out at once, the
cell's status becomes KKS_STATUS_TIMEOUT, the block still waits (bounded) for
its copies in flight, and the run stops after that attempt. The host reports
it as KksError; the device context stays usable, and a fresh run on the same
device afterwards matches the oracle.
"""

import numpy as np
import pytest

from conftest import copy_state, rel_l2

pytestmark = pytest.mark.gpu


def _case():
    from pf_kks_gpu import workloads
    from pf_kks_gpu.generator import MicrostructureSpec

    cfg = workloads.base_config(nx=64, ny=48, n_steps=8, n_map_saves=2, n_surface_samples=4)
    spec = MicrostructureSpec(64, 48, n_cells=3, n_particles=6, seed=5)
    return cfg, workloads.initial_state(cfg, spec)


def test_bounded_wait_timeout_reaches_the_host(tmp_path):
    from oracle import kks_oracle
    from pf_kks_gpu import _lib as L
    from pf_kks_gpu import solver
    from pf_kks_gpu.materials import MaterialTables

    cfg, state = _case()
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    cell = solver.Cell(cfg, tables, precision="mixed")
    try:
        assert cell.pipeline()[0], "64 x 48 should run the fused passes"
        cell.upload(*state)
        cell.set_wait_polls(0)
        status = cell.run(5)
        assert status == L.KKS_STATUS_TIMEOUT
        s = cell.state()
        assert s.attempts == 1 and s.istep <= 1  # the run stopped after the attempt that timed out
        with pytest.raises(L.KksError, match="bounded device wait ran out"):
            solver.raise_for_status(cell, status)
        assert cell.run(3) == L.KKS_STATUS_TIMEOUT  # the status is sticky until the state is reset
        # the same cell, default polls, state uploaded again: runs normally
        cell.set_wait_polls(-1)
        cell.upload(*state)
        assert cell.run(cfg.n_steps) == L.KKS_STATUS_OK
        again = cell.download()
    finally:
        cell.close()
    # a fresh run on the device afterwards
    fresh = solver.run(cfg, *copy_state(state), out_dir=str(tmp_path / "gpu"), verbose=False, precision="mixed")
    ref = kks_oracle.run(cfg, *copy_state(state), cfg.material_tables, out_dir=str(tmp_path / "cpu"))
    for name, a in zip(("eta", "X"), again[:2]):
        assert rel_l2(a, getattr(ref, name)) <= 1e-6, name
        assert rel_l2(getattr(fresh, name), getattr(ref, name)) <= 1e-6, name
        np.testing.assert_array_equal(a, getattr(fresh, name))


def test_wait_polls_needs_fused_passes():
    from pf_kks_gpu import _lib as L
    from pf_kks_gpu import solver
    from pf_kks_gpu.materials import MaterialTables

    cfg, state = _case()
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    cell = solver.Cell(cfg, tables, precision="fp64")
    try:
        with pytest.raises(L.KksError, match="nothing waits"):
            cell.set_wait_polls(0)
    finally:
        cell.close()
