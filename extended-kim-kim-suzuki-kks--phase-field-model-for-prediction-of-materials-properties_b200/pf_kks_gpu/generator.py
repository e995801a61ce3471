"""Seeded synthetic microstructures for the benchmark workloads.

The reference only places sharp circles read from a file
(``pf_kks/microstructure.py:7-52``). The workloads this package is measured on
need a different initial state, written here from scratch:

* a periodic Voronoi tessellation of the box with ``n_cells`` seeds drawn
  uniformly (minimum-image distance);
* ``n_particles`` circular Si particles centred on points drawn uniformly
  among the Voronoi edge pixels (plus a sub-pixel jitter), radius
  ``U(r_min, r_max)`` cells;
* a diffuse order parameter ``eta = max_p 1/2 [1 - tanh((r - R_p)/w)]`` with
  ``w`` chosen so that ``eta`` goes from 0.05 to 0.95 over ``width_cells``
  cells (periodic distance);
* Si fraction 1.0 in the particles and ``x_matrix + U(-noise, noise)`` in the
  matrix, blended by eta: ``X = eta x_particle + (1 - eta) X_matrix``;
* phase compositions from the closed KKS form at the initial temperature
  (``pf_kks/free_energy.py:74-95``), so that the state is KKS-consistent.

Every draw comes from ``numpy.random.Generator(PCG64(seed))`` in a fixed order,
so a (size, seed, parameters) triple always gives the same arrays.
"""

from dataclasses import dataclass

import numpy as np


@dataclass
class MicrostructureSpec:
    nx: int
    ny: int
    n_cells: int
    n_particles: int
    r_min: float = 3.0
    r_max: float = 8.0
    seed: int = 0
    x_matrix: float = 0.05
    x_noise: float = 0.002
    x_particle: float = 1.0
    width_cells: float = 4.0


def _periodic_delta(a, n):
    """Minimum-image difference on a periodic axis of length n."""
    return a - n * np.round(a / n)


def voronoi_labels(nx, ny, seeds):
    """Nearest-seed label of every grid point, periodic metric."""
    xs = np.arange(nx, dtype=np.float64)[:, None]
    ys = np.arange(ny, dtype=np.float64)[None, :]
    best = np.full((nx, ny), np.inf)
    label = np.zeros((nx, ny), dtype=np.int32)
    for i, (sx, sy) in enumerate(seeds):
        d2 = _periodic_delta(xs - sx, nx) ** 2 + _periodic_delta(ys - sy, ny) ** 2
        closer = d2 < best
        best = np.where(closer, d2, best)
        label = np.where(closer, i, label)
    return label


def voronoi_edges(label):
    """Pixels whose right or lower periodic neighbour carries another label."""
    return (label != np.roll(label, -1, axis=0)) | (label != np.roll(label, -1, axis=1))


def diffuse_eta(nx, ny, centres, radii, width_cells):
    """max over particles of 1/2 [1 - tanh((r - R)/w)], stamped in a local
    periodic window around each particle."""
    w = width_cells / (2.0 * np.arctanh(0.9))
    eta = np.zeros((nx, ny))
    for (cx, cy), R in zip(centres, radii):
        reach = int(np.ceil(R + 8.0 * w)) + 1
        ix = np.arange(int(np.floor(cx)) - reach, int(np.floor(cx)) + reach + 1)
        iy = np.arange(int(np.floor(cy)) - reach, int(np.floor(cy)) + reach + 1)
        dxs = (ix - cx)[:, None]
        dys = (iy - cy)[None, :]
        r = np.sqrt(dxs**2 + dys**2)
        prof = 0.5 * (1.0 - np.tanh((r - R) / w))
        gx = np.mod(ix, nx)[:, None]
        gy = np.mod(iy, ny)[None, :]
        if len(ix) > nx or len(iy) > ny:
            # A particle wider than the box: fold the window point by point.
            for a in range(len(ix)):
                for b in range(len(iy)):
                    eta[gx[a, 0], gy[0, b]] = max(eta[gx[a, 0], gy[0, b]], prof[a, b])
        else:
            eta[gx, gy] = np.maximum(eta[gx, gy], prof)
    return eta


def _phase_constants(A_alp, B_alp, A_thet, B_thet):
    return (B_alp - B_thet) / (2 * A_thet), A_alp / A_thet


def generate_on_device(cell, spec, A_alp, B_alp, A_thet, B_thet):
    """The state of :func:`generate`, written by the device into ``cell``
    (a :class:`pf_kks_gpu.solver.Cell` of the spec's size).

    The host draws what is per seed or per particle, in the same order and
    from the same stream as :func:`generate`; labels, edge pixels, the
    particles' profiles, the per-point matrix noise (the stream's next nx*ny
    doubles, drawn on the device from the generator state after the radii) and
    the phase compositions are computed on the device. Returns the number of
    edge pixels.
    """
    if (cell.nx, cell.ny) != (spec.nx, spec.ny):
        raise ValueError(f"cell is {cell.nx}x{cell.ny}, spec is {spec.nx}x{spec.ny}")
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    nx, ny = spec.nx, spec.ny
    seeds = rng.uniform(0.0, 1.0, size=(spec.n_cells, 2)) * np.array([nx, ny])
    n_edges = cell.voronoi_edges(seeds)
    pick = rng.integers(0, n_edges if n_edges else nx * ny, size=spec.n_particles)
    jitter = rng.uniform(-0.5, 0.5, size=(spec.n_particles, 2))
    radii = rng.uniform(spec.r_min, spec.r_max, size=spec.n_particles)
    w = spec.width_cells / (2.0 * np.arctanh(0.9))
    low, high = -spec.x_noise, spec.x_noise
    pc_shift, pc_ratio = _phase_constants(A_alp, B_alp, A_thet, B_thet)
    cell.generate_fields(pick, jitter, radii, w, spec.x_matrix, low, high - low, spec.x_particle,
                         rng.bit_generator.state, pc_shift, pc_ratio, picks_are_points=(n_edges == 0))
    return n_edges


def generate(spec, A_alp, B_alp, A_thet, B_thet):
    """Initial (eta, X, X_al, X_th), each (nx, ny, 1) float64.

    ``A_alp, B_alp, A_thet, B_thet`` are the parabola coefficients at the
    initial temperature (``MaterialTables.at(T0, ...)``).
    """
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    nx, ny = spec.nx, spec.ny
    seeds = rng.uniform(0.0, 1.0, size=(spec.n_cells, 2)) * np.array([nx, ny])
    edges = voronoi_edges(voronoi_labels(nx, ny, seeds))
    edge_idx = np.flatnonzero(edges.ravel())
    if edge_idx.size == 0:  # a single cell has no edge: spread particles uniformly
        edge_idx = np.arange(nx * ny)
    pick = rng.integers(0, edge_idx.size, size=spec.n_particles)
    px, py = np.divmod(edge_idx[pick], ny)
    jitter = rng.uniform(-0.5, 0.5, size=(spec.n_particles, 2))
    centres = np.stack([px + jitter[:, 0], py + jitter[:, 1]], axis=1)
    radii = rng.uniform(spec.r_min, spec.r_max, size=spec.n_particles)
    eta = diffuse_eta(nx, ny, centres, radii, spec.width_cells)
    x_mat = spec.x_matrix + rng.uniform(-spec.x_noise, spec.x_noise, size=(nx, ny))
    X = eta * spec.x_particle + (1.0 - eta) * x_mat
    eta = eta.reshape(nx, ny, 1)
    X = X.reshape(nx, ny, 1)
    h = 3.0 * eta**2 - 2 * eta**3
    X_al = (X - h * ((B_alp - B_thet) / (2 * A_thet))) / ((1 - h) + h * (A_alp / A_thet))
    X_th = (A_alp / A_thet) * X_al + (B_alp - B_thet) / (2 * A_thet)
    return eta, X, X_al, X_th
