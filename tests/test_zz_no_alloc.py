"""The allocation-free entry point kks_state_sums_noalloc, through the C ABI.

It serves callers that cannot allocate device memory (a framework that owns
all device memory through its own pool, or a latency-critical loop that must
not call cudaMalloc / cudaFree, which may synchronise the device): they pass
their own device buffers and the library uses only a fixed scratch array.
The test allocates the state buffers itself (with torch), as such a caller
would, and checks two calls in a row (different grid sizes, so the second call
runs on scratch left over from the first) against the old-state histories that
the step's own entry point (kks_run) reports for the same states.
"""

import ctypes

import numpy as np
import pytest

from conftest import copy_state

pytestmark = pytest.mark.gpu


def _step_histories(cfg, state):
    """Histories of the first step from kks_run: they describe the input state."""
    from pf_kks_gpu import solver
    from pf_kks_gpu._lib import H
    from pf_kks_gpu.materials import MaterialTables

    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    cell = solver.Cell(cfg, tables, precision="fp64")
    try:
        cell.upload(*copy_state(state))
        assert cell.run(1) == 0
        _, rows = cell.drain()
    finally:
        cell.close()
    row = rows[0]
    surf_old = row[H["surf"]] - row[H["dsurf"]]  # step 1 is always a surface step
    return row[H["eta_mean"]], row[H["X_al_mean"]], row[H["X_th_mean"]], surf_old


def _noalloc_sums(lib, eta_dev, X_dev, nx, ny, out_dev):
    import torch

    out_dev.fill_(float("nan"))  # every slot must be written by the call
    torch.cuda.synchronize()
    rc = lib.kks_state_sums_noalloc(ctypes.c_void_p(eta_dev.data_ptr()), ctypes.c_void_p(X_dev.data_ptr()), nx, ny,
                                    ctypes.c_void_p(out_dev.data_ptr()), None)
    assert rc == 0, lib.kks_last_error()
    torch.cuda.synchronize()
    return out_dev.cpu().numpy()


def test_state_sums_noalloc_match_step_histories():
    import torch

    from pf_kks_gpu import _lib, workloads
    from pf_kks_gpu.generator import MicrostructureSpec

    lib = _lib.load()
    out_dev = torch.empty(6, dtype=torch.float64, device="cuda")
    cases = [
        (workloads.demo160(n_steps=2)[0], MicrostructureSpec(160, 160, n_cells=4, n_particles=40, seed=0)),
        (workloads.base_config(nx=96, ny=80, n_steps=2), MicrostructureSpec(96, 80, n_cells=3, n_particles=9, seed=4)),
    ]
    for cfg, spec in cases:  # two calls in a row
        state = workloads.initial_state(cfg, spec)
        eta_mean, x_al_mean, x_th_mean, surf_old = _step_histories(cfg, state)
        nx, ny = cfg.nx, cfg.ny
        eta_dev = torch.from_numpy(np.ascontiguousarray(state[0].reshape(nx, ny))).cuda()
        X_dev = torch.from_numpy(np.ascontiguousarray(state[1].reshape(nx, ny))).cuda()
        s = _noalloc_sums(lib, eta_dev, X_dev, nx, ny, out_dev)
        assert np.all(np.isfinite(s))
        assert s[0] / (nx * ny) == pytest.approx(eta_mean, rel=1e-12)
        assert s[1] / s[2] == pytest.approx(x_al_mean, rel=1e-12)
        assert s[3] / s[4] == pytest.approx(x_th_mean, rel=1e-12)
        assert s[5] * (cfg.dx**2 / (2 * cfg.lambd)) == pytest.approx(surf_old, rel=1e-12)


def test_state_sums_noalloc_rejects_oversized_grids():
    import torch

    from pf_kks_gpu import _lib

    lib = _lib.load()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    rc = lib.kks_state_sums_noalloc(p, p, 1 << 14, 1 << 13, p, None)  # 2^27 points > 2^26
    assert rc == -5 and b"KKS_NOALLOC_MAX_POINTS" in lib.kks_last_error()
    assert lib.kks_state_sums_noalloc(None, p, 8, 8, p, None) == -1
