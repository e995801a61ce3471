"""Initial state written on the device (csrc/kks_init.cu through the C ABI).

* The synthetic microstructure: against the host generator on the same seed:
  the same edge-pixel count, the matrix noise bit for bit (X where no particle
  window reaches), eta and X within a few ulp (the device's tanh is not
  numpy's), the phase compositions within 1e-13 relative or 4e-15 absolute
  (FP64 state; X_al crosses 0 in the particles) or 1 float ulp (the FP32
  X_al / X_th of the mixed path). Sizes from a
  tessellation without edges and a particle wider than the box up to the
  1420^2 workload.
* Sharp precipitates and nuclei: bit for bit against the reference's numba
  functions (tests/golden/reference_init.npz).
* Nucleus insertion at ranked candidates, and the history columns that the
  nucleation coupling reads.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu


def _setup(nx, ny, precision="fp64", n_steps=4, **kw):
    from pf_kks_gpu import solver, workloads
    from pf_kks_gpu.materials import MaterialTables

    cfg = workloads.base_config(nx=nx, ny=ny, n_steps=n_steps, **kw)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    cell = solver.Cell(cfg, tables, precision=precision, device=0)
    T0 = float(np.interp(0, np.array(cfg.schedule_time), np.array(cfg.schedule_temperature)))
    coefs = [float(tables.at(T0, n)) for n in ("A_alp", "B_alp", "A_thet", "B_thet")]
    return cfg, tables, cell, coefs


def _edge_count(spec):
    from pf_kks_gpu.generator import voronoi_edges, voronoi_labels

    rng = np.random.Generator(np.random.PCG64(spec.seed))
    seeds = rng.uniform(0.0, 1.0, size=(spec.n_cells, 2)) * np.array([spec.nx, spec.ny])
    return int(voronoi_edges(voronoi_labels(spec.nx, spec.ny, seeds)).sum())


CASES = [
    (96, 80, 5, 12, 8.0),  # several cells, particles across the box edges
    (64, 64, 1, 6, 8.0),  # one cell: no edge pixels, particles anywhere
    (24, 20, 2, 3, 16.0),  # particles wider than the box (folded windows)
    (160, 160, 4, 40, 8.0),  # the 160^2 workload's sizes
]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nx,ny,cells,parts,rmax", CASES)
def test_device_generator_matches_host(precision, nx, ny, cells, parts, rmax):
    from pf_kks_gpu.generator import MicrostructureSpec, generate, generate_on_device

    cfg, tables, cell, coefs = _setup(nx, ny, precision)
    try:
        spec = MicrostructureSpec(nx, ny, n_cells=cells, n_particles=parts, r_min=3, r_max=rmax, seed=3)
        host = generate(spec, *coefs)
        n_edges = generate_on_device(cell, spec, *coefs)
        assert n_edges == _edge_count(spec)
        dev = cell.download()
    finally:
        cell.close()
    _compare(host, dev, precision, require_outside=(nx, ny) != (24, 20))


def _compare(host, dev, precision, require_outside=True):
    eta_h, X_h, Xal_h, Xth_h = (a.reshape(-1) for a in host)
    eta_d, X_d, Xal_d, Xth_d = (a.reshape(-1) for a in dev)
    assert np.max(np.abs(eta_d - eta_h)) <= 1e-15
    outside = eta_h == 0.0
    assert outside.any() or not require_outside  # the folded windows of the 24 x 20 case cover the whole box
    assert np.array_equal(eta_d[outside], eta_h[outside])
    assert np.array_equal(X_d[outside], X_h[outside])  # the PCG64 noise, bit for bit
    assert np.max(np.abs(X_d - X_h)) <= 1e-15
    if precision == "fp64":
        # X_al crosses 0 inside the particles: an ulp of eta or X there is an absolute, not relative, error
        np.testing.assert_allclose(Xal_d, Xal_h, rtol=1e-13, atol=4e-15)
        np.testing.assert_allclose(Xth_d, Xth_h, rtol=1e-13, atol=4e-15)
    else:
        for d, h in ((Xal_d, Xal_h), (Xth_d, Xth_h)):
            ulp = np.spacing(np.abs(h.astype(np.float32))).astype(np.float64)
            assert np.all(np.abs(d - h.astype(np.float32).astype(np.float64)) <= ulp)


def test_device_generator_at_1420():
    from pf_kks_gpu import workloads
    from pf_kks_gpu.generator import generate_on_device

    cfg, spec = workloads.ramp1420(n_steps=4)
    _, tables, cell, coefs = _setup(1420, 1420, "mixed", n_steps=4, schedule_time=cfg.schedule_time,
                                     schedule_temperature=cfg.schedule_temperature)
    try:
        host = workloads.initial_state(cfg, spec)
        assert generate_on_device(cell, spec, *coefs) == _edge_count(spec)
        dev = cell.download()
    finally:
        cell.close()
    _compare(host, dev, "mixed")


def test_run_from_device_state_matches_run_from_upload():
    from pf_kks_gpu.generator import MicrostructureSpec, generate, generate_on_device

    spec = MicrostructureSpec(64, 64, n_cells=3, n_particles=10, seed=5)
    out = []
    for on_device in (False, True):
        cfg, tables, cell, coefs = _setup(64, 64, "fp64", n_steps=6)
        try:
            if on_device:
                generate_on_device(cell, spec, *coefs)
            else:
                cell.upload(*generate(spec, *coefs))
            assert cell.run(6) == 0
            out.append(cell.download())
        finally:
            cell.close()
    for a, b in zip(*out):
        assert rel_l2(a, b) <= 1e-13


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLDEN, "reference_init.npz"))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_place_precipitates_and_nuclei_match_reference(gold, precision):
    from pf_kks_gpu.microstructure import add_nuclei_on_device, place_precipitates_on_device

    nx, ny, nz = (int(v) for v in gold["place_grid"])
    dx = float(gold["place_dx"])
    xm, xp = float(gold["place_xm"]), float(gold["place_xp"])
    cfg, tables, cell, _ = _setup(nx, ny, precision)
    r32 = (lambda a: a) if precision == "fp64" else (lambda a: np.asarray(a, np.float32).astype(np.float64))
    try:
        place_precipitates_on_device(cell, nx, ny, nz, dx, dx, dx, xm, xp, gold["place_r"], gold["place_ox"],
                                     gold["place_oy"], gold["place_oz"])
        eta, X, X_al, X_th = (a.reshape(-1) for a in cell.download())
        inside = np.unpackbits(gold["place_mask"])[: nx * ny].astype(bool)
        assert np.array_equal(eta, np.where(inside, 1.0, 0.0))
        assert np.array_equal(X, np.where(inside, xp, xm))
        assert np.array_equal(X_al, r32(np.where(inside, 0.0, xm)))
        assert np.array_equal(X_th, r32(np.where(inside, xp, 0.0)))
        add_nuclei_on_device(cell, nx, ny, nz, dx, dx, dx, gold["nuc_r"], gold["nuc_ox"], gold["nuc_oy"],
                             gold["nuc_oz"])
        eta, X, X_al, X_th = (a.reshape(-1) for a in cell.download())
        nuc = np.unpackbits(gold["nuclei_mask"])[: nx * ny].astype(bool)
        assert np.array_equal(X == 0.99999, nuc)
        assert np.array_equal(eta == 1.0, np.unpackbits(gold["after_eta_mask"])[: nx * ny].astype(bool))
        assert np.array_equal(X_al[nuc], np.zeros(nuc.sum()))
        assert np.array_equal(X_th[nuc], r32(np.full(nuc.sum(), 0.99999)))
    finally:
        cell.close()


def test_insert_nuclei_at_ranked_candidates():
    from pf_kks_gpu import nucleation as NU
    from pf_kks_gpu.generator import MicrostructureSpec, generate_on_device

    spec = MicrostructureSpec(150, 130, n_cells=4, n_particles=30, seed=8)
    cfg, tables, cell, coefs = _setup(150, 130, "fp64")
    try:
        generate_on_device(cell, spec, *coefs)
        eta0 = cell.download()[0].reshape(-1)
        cand = np.flatnonzero(eta0 < 0.05)
        assert cell.count_below(0.05) == cand.size
        ranks = np.array([0, 1, 777, cand.size // 2, cand.size - 1])
        cell.insert_nuclei(ranks, 0.05)
        eta1 = cell.download()[0].reshape(-1)
        want = eta0.copy()
        want[cand[ranks]] = 1.0
        assert np.array_equal(eta1, want)
        # the reference's random draw, on the device
        rank = NU.insert_random_nucleus_on_device(cell, np.random.RandomState(4))
        cand1 = np.flatnonzero(eta1 < 0.05)
        want[cand1[rank]] = 1.0
        host = eta1.copy()
        NU.insert_random_nucleus(cand1, host, np.random.RandomState(4))
        assert np.array_equal(host, want)
        assert np.array_equal(cell.download()[0].reshape(-1), want)
        with pytest.raises(Exception):
            cell.insert_nuclei([cand1.size + 5], 0.05)
    finally:
        cell.close()


def test_history_rows_carry_diffusivity_and_vacancies_for_nucleation():
    from pf_kks_gpu import nucleation as NU
    from pf_kks_gpu._lib import H
    from pf_kks_gpu.generator import MicrostructureSpec, generate_on_device

    spec = MicrostructureSpec(64, 64, n_cells=2, n_particles=6, seed=1)
    cfg, tables, cell, coefs = _setup(64, 64, "fp64", n_steps=8)
    try:
        generate_on_device(cell, spec, *coefs)
        assert cell.run(8) == 0
        _, rows = cell.drain()
        assert rows.shape[0] == 8
        assert np.all(rows[:, H["D"]] > 0)
        assert rows[-1, H["Xv"]] == cell.state().Xv
        coupling = NU.NucleationCoupling(cfg, tables, B=1e-3, X_al_eq=0.0)
        n = [coupling.increment(r) for r in rows]
        assert all(np.isfinite(v) and v >= 0 for v in n)
        coupling.expected = 1.5  # owe one nucleus
        assert coupling.after_run(cell, rows[:0]) == 1
        assert len(coupling.inserted) == 1
    finally:
        cell.close()
