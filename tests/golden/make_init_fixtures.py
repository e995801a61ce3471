"""Generate ``reference_init.npz`` from the reference itself: the initial-state
and nucleation functions that the device versions are checked against.

    NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_init_fixtures.py [REF]

REF (the argument, or $PF_KKS_REFERENCE) is read, never written. Contents:

* ``place_*``: ``pf_kks.microstructure.place_precipitates`` (numba,
  pf_kks/microstructure.py:7-52) on a 96 x 80 x 1 grid with circles that cross
  the box edges, overlap, and one of radius 0; then ``add_nuclei``
  (pf_kks/microstructure.py:55-74) on that state. Each output field takes two
  values, so it is stored as a packed mask plus the inputs.
* ``nuc_args`` / ``nuc_out``: ``pf_kks.nucleation.nucleation_increment``
  (pf_kks/nucleation.py:15-98) on a grid of temperatures, matrix fractions,
  box shapes and heterogeneous factors, with the parabola coefficients and
  interface energy of final_export.npz at each temperature.
* ``ins_*``: ``pf_kks.nucleation.insert_random_nucleus`` (pf_kks/nucleation.py:103-111)
  with ``numpy.random.RandomState(seed)`` on candidate lists.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    sys.path.insert(0, ref)
    from pf_kks import microstructure as M
    from pf_kks import nucleation as NU

    out = {}
    nx, ny, nz = 96, 80, 1
    dx = 0.5e-9
    rng = np.random.Generator(np.random.PCG64(77))
    n = 14
    ox = rng.uniform(-4, nx + 4, n) * dx
    oy = rng.uniform(-4, ny + 4, n) * dx
    oz = np.zeros(n)
    r = rng.uniform(2, 12, n) * dx
    r[3] = 0.0
    ox[5], oy[5], r[5] = ox[4] + 2 * dx, oy[4], r[4]  # overlapping pair
    eta, X, X_mat, X_pre = M.place_precipitates(nx, ny, nz, dx, dx, dx, 0.02, 0.98, r, ox, oy, oz)
    out.update(place_grid=np.array([nx, ny, nz]), place_dx=dx, place_xm=0.02, place_xp=0.98, place_r=r,
               place_ox=ox, place_oy=oy, place_oz=oz)
    out["place_mask"] = np.packbits((eta[..., 0] == 1).ravel())
    assert np.array_equal(X[..., 0], np.where(eta[..., 0] == 1, 0.98, 0.02))
    assert np.array_equal(X_mat[..., 0], np.where(eta[..., 0] == 1, 0.0, 0.02))
    assert np.array_equal(X_pre[..., 0], np.where(eta[..., 0] == 1, 0.98, 0.0))
    m = 6
    nox = rng.uniform(0, nx, m) * dx
    noy = rng.uniform(0, ny, m) * dx
    noz = np.zeros(m)
    nr = rng.uniform(1, 4, m) * dx
    M.add_nuclei(nx, ny, nz, dx, dx, dx, eta, X, X_mat, X_pre, nr, nox, noy, noz)
    out.update(nuc_r=nr, nuc_ox=nox, nuc_oy=noy, nuc_oz=noz)
    out["nuclei_mask"] = np.packbits((X[..., 0] == 0.99999).ravel())
    out["after_eta_mask"] = np.packbits((eta[..., 0] == 1).ravel())

    d = np.load(os.path.join(ref, "data", "inputs", "final_export.npz"))
    args, res = [], []
    for T in (420.0, 450.0, 500.0, 560.0, 640.0):
        coeffs = [float(np.interp(T, d["T"], d[k])) for k in ("A_fcc", "B_fcc", "C_fcc", "A_dia", "B_dia", "C_dia")]
        sigma = float(np.interp(T, d["T"], d["gamma"]))
        for X_al_mean in (0.004, 0.012, 0.02, 0.03):
            for grid, B in (((64, 64, 1), 1e-3), ((32, 1, 1), 1e-2), ((16, 16, 16), 1e-3), ((128, 96, 1), 5e-4)):
                a = (B, 0.005, 12.0, 0.5, T, 0.5e-9, 0.5e-9, 0.5e-9, *grid, 1e-18, *coeffs, sigma, X_al_mean, 1e-5)
                args.append([float(v) for v in a])
                res.append([float(v) for v in NU.nucleation_increment(*a)])
    out["nuc_args"] = np.array(args)
    out["nuc_out"] = np.array(res)

    picks = []
    for seed, size in ((0, 10), (1, 500), (2, 7777)):
        cand = np.flatnonzero(np.random.RandomState(seed + 100).uniform(size=2 * size) < 0.5)
        e = np.zeros(2 * size)
        NU.insert_random_nucleus(cand, e, np.random.RandomState(seed))
        picks.append([seed, 2 * size, len(cand), int(np.flatnonzero(e == 1)[0])])
    out["ins_cases"] = np.array(picks)
    path = os.path.join(HERE, "reference_init.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    _ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PF_KKS_REFERENCE")
    if not _ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_CHECKOUT (or set PF_KKS_REFERENCE)")
    main(_ref)
