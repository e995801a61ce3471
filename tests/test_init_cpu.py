"""Initial state and nucleation on the CPU (no GPU):

* the host mirrors of ``place_precipitates`` / ``add_nuclei`` /
  ``nucleation_increment`` / ``insert_random_nucleus`` against fixtures made
  by the reference itself (tests/golden/make_init_fixtures.py);
* the algorithms of the device generator (csrc/kks_init.cu) restated in
  Python and checked against numpy's: the PCG64 jump-ahead that draws the
  matrix noise point by point, the periodic-window images behind eta, and the
  chunked ordered selection of edge pixels.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN

from pf_kks_gpu import microstructure as MS
from pf_kks_gpu import nucleation as NU
from pf_kks_gpu.generator import MicrostructureSpec, diffuse_eta, generate, voronoi_edges, voronoi_labels


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLDEN, "reference_init.npz"))


def _mask(packed, n):
    return np.unpackbits(packed)[:n].astype(bool)


def test_place_precipitates_and_add_nuclei_match_reference(gold):
    nx, ny, nz = (int(v) for v in gold["place_grid"])
    dx = float(gold["place_dx"])
    xm, xp = float(gold["place_xm"]), float(gold["place_xp"])
    eta, X, X_mat, X_pre = MS.place_precipitates(nx, ny, nz, dx, dx, dx, xm, xp, gold["place_r"], gold["place_ox"],
                                                  gold["place_oy"], gold["place_oz"])
    inside = _mask(gold["place_mask"], nx * ny).reshape(nx, ny)
    assert inside.any() and not inside.all()
    assert np.array_equal(eta[..., 0] == 1, inside)
    assert np.array_equal(X[..., 0], np.where(inside, xp, xm))
    assert np.array_equal(X_mat[..., 0], np.where(inside, 0.0, xm))
    assert np.array_equal(X_pre[..., 0], np.where(inside, xp, 0.0))
    MS.add_nuclei(nx, ny, nz, dx, dx, dx, eta, X, X_mat, X_pre, gold["nuc_r"], gold["nuc_ox"], gold["nuc_oy"],
                  gold["nuc_oz"])
    assert np.array_equal((X[..., 0] == 0.99999).ravel(), _mask(gold["nuclei_mask"], nx * ny))
    assert np.array_equal((eta[..., 0] == 1).ravel(), _mask(gold["after_eta_mask"], nx * ny))


def test_nucleation_increment_matches_reference(gold):
    args, ref = gold["nuc_args"], gold["nuc_out"]
    assert (ref[:, 0] > 0).any() and (ref[:, 0] == 0).any()
    for a, r in zip(args, ref):
        a = list(a)
        for k in (8, 9, 10):  # grid sizes
            a[k] = int(a[k])
        n, rc = NU.nucleation_increment(*a)
        assert float(n) == r[0] and float(rc) == r[1], (a, n, rc, r)


def test_insert_random_nucleus_matches_reference(gold):
    for seed, size, n_cand, where in gold["ins_cases"]:
        cand = np.flatnonzero(np.random.RandomState(seed + 100).uniform(size=size) < 0.5)
        assert cand.size == n_cand
        e = np.zeros(size)
        NU.insert_random_nucleus(cand, e, np.random.RandomState(seed))
        assert np.flatnonzero(e == 1).tolist() == [where]


# -- the device generator's algorithms, restated ----------------------------

MULT = (0x2360ED051FC65DA4 << 64) | 0x4385DF649FCCF645
M128 = (1 << 128) - 1


def lcg_jump(d, inc):
    """(mult, plus) of d LCG steps, by squaring (the kernel's lcg_jump)."""
    cm, cp, am, ap = MULT, inc, 1, 0
    while d:
        if d & 1:
            am, ap = (am * cm) & M128, (ap * cm + cp) & M128
        cp = ((cm + 1) * cp) & M128
        cm = (cm * cm) & M128
        d >>= 1
    return am, ap


def pcg_output(s):
    x = ((s >> 64) ^ s) & ((1 << 64) - 1)
    rot = s >> 122
    return ((x >> rot) | (x << ((64 - rot) & 63))) & ((1 << 64) - 1)


def device_noise(state, inc, n, low, rng_range, threads):
    """Point i of thread g = i mod G: state jumped g + 1 steps, then G at a time."""
    out = np.empty(n)
    gm, gp = lcg_jump(threads, inc)
    for g in range(min(threads, n)):
        am, ap = lcg_jump(g + 1, inc)
        s = (am * state + ap) & M128
        for i in range(g, n, threads):
            out[i] = low + rng_range * ((pcg_output(s) >> 11) * (1.0 / 9007199254740992.0))
            s = (gm * s + gp) & M128
    return out


@pytest.mark.parametrize("threads", [1, 7, 256])
def test_pcg64_jump_ahead_reproduces_numpy_noise(threads):
    spec = MicrostructureSpec(23, 17, n_cells=3, n_particles=5, seed=4)
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    rng.uniform(size=(spec.n_cells, 2))
    rng.integers(0, 50, size=spec.n_particles)  # 32-bit draws leave a buffered half word; next_double skips it
    rng.uniform(-0.5, 0.5, size=(spec.n_particles, 2))
    rng.uniform(3, 8, size=spec.n_particles)
    st = rng.bit_generator.state["state"]
    low, high = -spec.x_noise, spec.x_noise
    want = rng.uniform(low, high, size=spec.nx * spec.ny)
    got = device_noise(st["state"], st["inc"], spec.nx * spec.ny, low, high - low, threads)
    assert np.array_equal(got, want)


def window_eta(nx, ny, centres, radii, width_cells):
    """eta by the kernel's per-point rule: every image ix = gx (mod nx) inside
    the window [floor(c) - reach, floor(c) + reach] of each particle."""
    w = width_cells / (2.0 * np.arctanh(0.9))
    eta = np.zeros((nx, ny))
    for (cx, cy), R in zip(centres, radii):
        reach = int(np.ceil(R + 8.0 * w)) + 1
        xlo, ylo = int(np.floor(cx)) - reach, int(np.floor(cy)) - reach
        length = 2 * reach + 1
        for gx in range(nx):
            ixs = range(xlo + (gx - xlo) % nx, xlo + length, nx)
            for gy in range(ny):
                for ix in ixs:
                    dxs = np.float64(ix) - cx
                    for iy in range(ylo + (gy - ylo) % ny, ylo + length, ny):
                        dys = np.float64(iy) - cy
                        r = np.sqrt(dxs * dxs + dys * dys)
                        eta[gx, gy] = max(eta[gx, gy], 0.5 * (1.0 - np.tanh((r - R) / w)))
    return eta


def test_window_images_reproduce_host_stamping():
    # a particle wider than the box (folded windows) and ordinary ones
    centres = np.array([[3.2, 17.9], [11.5, 0.3], [20.0, 9.0]])
    radii = np.array([2.5, 14.0, 4.0])
    nx, ny = 24, 20
    want = diffuse_eta(nx, ny, centres, radii, 4.0)
    got = window_eta(nx, ny, centres, radii, 4.0)
    assert np.array_equal(got, want)


def chunked_select(mask, ranks, chunk=1024):
    """The kernel's ordered selection: per-chunk counts, exclusive scan, then
    the rank's chunk scanned in order."""
    flat = mask.ravel()
    nchunks = -(-flat.size // chunk)
    counts = np.array([flat[c * chunk:(c + 1) * chunk].sum() for c in range(nchunks)])
    off = np.concatenate([[0], np.cumsum(counts)])
    out = []
    for r in ranks:
        c = int(np.searchsorted(off, r, side="right") - 1)
        local = r - off[c]
        idx = np.flatnonzero(flat[c * chunk:(c + 1) * chunk])[local]
        out.append(c * chunk + idx)
    return np.array(out), int(off[-1])


def test_chunked_selection_is_flatnonzero():
    labels = voronoi_labels(70, 50, np.array([[3.0, 4.0], [40.2, 33.3], [66.6, 10.0], [20.0, 45.0]]))
    edges = voronoi_edges(labels)
    ranks = np.random.default_rng(3).integers(0, edges.sum(), size=64)
    got, total = chunked_select(edges, ranks)
    assert total == edges.sum()
    assert np.array_equal(got, np.flatnonzero(edges.ravel())[ranks])


def test_host_generator_determinism_and_ranges():
    spec = MicrostructureSpec(40, 36, n_cells=3, n_particles=6, seed=9)
    a = generate(spec, 1.0, -0.1, 2.0, -0.2)
    b = generate(spec, 1.0, -0.1, 2.0, -0.2)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    assert 0.0 <= a[0].min() and a[0].max() <= 1.0
