"""The bounds-check debug build (libkks_b200_check.so, -DKKS_BOUNDS_CHECK).

The fused passes of that build check, per block, the rows or columns it works
on against the grid, its partial-sum row against the buffer and its sequences
against the launch's shared memory, and record the first failure instead of
faulting (csrc/kks_check.cuh). Here the debug build runs, in a child process
(KKS_LIBRARY selects the library), a mixed cell on the fused passes at 100 x 80
and at 1420^2 (prime-71 passes, tensor copies), the same cells with every
column tile, and a batch: no check may fail, and the results must equal the
release build's within the mixed path's bar.
"""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import PKG, REPO

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, os, sys
sys.path.insert(0, os.environ["KKS_TEST_PKG"])
import numpy as np
from pf_kks_gpu import _lib as L, solver, workloads
from pf_kks_gpu.ensemble import Ensemble
from pf_kks_gpu.generator import MicrostructureSpec
from pf_kks_gpu.materials import MaterialTables

out = {}
checked, first = L.bounds_report(0)
out["checked"] = checked
sums = {}
for (nx, ny, npart, steps) in ((100, 80, 12, 6), (1420, 1420, 1200, 2)):
    cfg = workloads.base_config(nx=nx, ny=ny, n_steps=steps, n_map_saves=2, n_surface_samples=steps)
    spec = MicrostructureSpec(nx, ny, n_cells=40 if nx > 1000 else 3, n_particles=npart, seed=9)
    state = workloads.initial_state(cfg, spec)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    for cols in (1, 2, 3, 4):
        cell = solver.Cell(cfg, tables, precision="mixed")
        assert cell.pipeline()[0]
        shape = cell.launch_shape()
        cell.set_launch_shape(1, cols, shape["field_blocks"])
        cell.upload(*state)
        assert cell.run(steps) == 0
        e, x, _, _ = cell.download()
        cell.close()
        sums[f"{nx}x{ny}/{cols}"] = [e.ravel().tolist()[::97], x.ravel().tolist()[::97]]
members = []
for k, n in enumerate((128, 192, 256)):
    cfg = workloads.base_config(nx=n, ny=n, n_steps=5, n_map_saves=2, n_surface_samples=5)
    spec = MicrostructureSpec(n, n, n_cells=3, n_particles=20, seed=40 + k)
    members.append((cfg, workloads.initial_state(cfg, spec)))
ens = Ensemble(members, precision="mixed", batched=True)
ens.run(5)
for k, c in enumerate(ens.cells):
    e, x, _, _ = c.download()
    sums[f"batch{k}"] = [e.ravel().tolist()[::97], x.ravel().tolist()[::97]]
ens.close()
checked, first = L.bounds_report(0)
out["checked_after"] = checked
out["first"] = first
out["sums"] = sums
print("RESULT" + json.dumps(out))
"""


def _child(lib):
    env = dict(os.environ)
    env["KKS_TEST_PKG"] = PKG
    if lib:
        env["KKS_LIBRARY"] = lib
    else:
        env.pop("KKS_LIBRARY", None)
    run = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=900,
                         cwd=REPO)
    assert run.returncode == 0, run.stderr[-4000:]
    line = [x for x in run.stdout.splitlines() if x.startswith("RESULT")][-1]
    return json.loads(line[len("RESULT"):])


def test_bounds_check_build_records_nothing_and_matches_release():
    from pf_kks_gpu import _lib as L

    if not os.path.exists(L.CHECK_LIB_PATH):
        from pf_kks_gpu import build

        build.build(bounds_check=True)
    dbg = _child(L.CHECK_LIB_PATH)
    assert dbg["checked"] and dbg["checked_after"], "the child did not load the bounds-check build"
    assert dbg["first"] == 0, f"a bounds check failed: site {dbg['first'] >> 44}, index {dbg['first'] & ((1 << 44) - 1)}"
    rel = _child(None)
    assert not rel["checked"]
    for key, (e_dbg, x_dbg) in dbg["sums"].items():
        e_rel, x_rel = rel["sums"][key]
        for a, b in ((e_dbg, e_rel), (x_dbg, x_rel)):
            a, b = np.asarray(a), np.asarray(b)
            assert np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(b), key
