"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run in a checkout that has the reference package (``pf_kks``) at REF (given as the
argument or in $PF_KKS_REFERENCE; it is read, never written):

    NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_fixtures.py [REF]

It writes

* ``reference_small.npz`` + ``reference_small_logs.json``: ``pf_kks.solver.run``
  on the setups of the reference's equivalence tests
  (tests/test_solver_equivalence.py:79-118, conftest.py:19-51): fixed steps,
  relaxed state, accepted, enlarged, rejected + abort. Fields, every history,
  good_step, ttime, map names and the two log files.
* ``archived_735.npz``: the map archived by the 2022 reproducible run after
  its first step (data/reference/reproducible_run/map0.07s_400_400.00K.npz,
  used by tests/test_archived_run.py:35-46) reduced to 4096 sampled points and
  the sum / sum of squares of each field, its history keys, the first line of
  the archived dtime.txt and the first 20 archived history rows
  (data/histories/reproducible_run.npz, tests/test_archived_run.py:49-61).
* ``reference_demo160.npz``: ``pf_kks.solver.run`` for 20 steps on the 160 x 160
  synthetic microstructure of this package's generator (seed 0), reduced the
  same way.
"""

import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(REPO, "extended-kim-kim-suzuki-kks--phase-field-model-for-prediction-of-materials-properties_b200")

FIELDS = ("X", "X_al", "X_th", "eta")
HISTORIES = ("eta_mean", "deta_mean", "X_mean", "X_al_mean", "dX_al_mean", "X_th_mean", "dX_th_mean", "dT", "T",
             "dtime", "time", "time_s", "surf", "dsurf", "L", "energy_s", "dtime_s", "residual_total",
             "residual_energy_derivative", "residual_diffusion", "residual_allen_cahn", "residual_temperature")


def sample_index(n_total, k=4096, seed=1234):
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.sort(rng.choice(n_total, size=min(k, n_total), replace=False))


def summarize(prefix, fields, out):
    for name, a in fields.items():
        flat = np.asarray(a, dtype=np.float64).ravel()
        idx = sample_index(flat.size)
        out[f"{prefix}{name}_idx"] = idx
        out[f"{prefix}{name}_val"] = flat[idx]
        out[f"{prefix}{name}_sum"] = flat.sum()
        out[f"{prefix}{name}_sumsq"] = (flat * flat).sum()


def main(ref):
    sys.path.insert(0, ref)
    sys.path.insert(0, PKG)
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "numba_cache"))
    from pf_kks import solver
    from pf_kks.config import SimulationConfig
    from pf_kks.microstructure import place_precipitates

    from pf_kks_gpu import workloads

    tables = os.path.join(ref, "data", "inputs", "final_export.npz")

    def small(**kw):
        p = dict(nx=64, ny=64, n_steps=40, n_map_saves=3, n_surface_samples=10, material_tables=tables)
        p.update(kw)
        return SimulationConfig(**p)

    def three(cfg):
        dx = cfg.dx
        r = np.array([3e-9, 2e-9, 4e-9])
        ox = np.array([8e-9, 20e-9, cfg.nx * dx * 0.6])
        oy = np.array([10e-9, 22e-9, cfg.ny * dx * 0.3])
        return place_precipitates(cfg.nx, cfg.ny, cfg.nz, dx, dx, dx, cfg.x_matrix, cfg.x_precipitate, r, ox, oy,
                                  np.zeros(3))

    def cp(s):
        return tuple(np.array(a, copy=True) for a in s)

    out, logs = {}, {}
    tmp = tempfile.mkdtemp()

    def record(case, cfg, state):
        d = os.path.join(tmp, case)
        try:
            res = solver.run(cfg, *cp(state), out_dir=d, verbose=False)
            for name in FIELDS:
                out[f"{case}_{name}"] = getattr(res, name)
            for name in HISTORIES:
                out[f"{case}_h_{name}"] = np.asarray(res.history[name], dtype=np.float64)
            out[f"{case}_good_step"] = -1 if res.good_step is None else res.good_step
            out[f"{case}_ttime"] = res.ttime
            if case == "fixed40":
                out[f"{case}_sig_el"] = res.sig_el
                out[f"{case}_eps_el"] = res.eps_el
            err = ""
        except solver.AdaptiveStepError as exc:
            err = str(exc)
        logs[case] = {
            "error": err,
            "maps": sorted(os.listdir(os.path.join(d, "saved_maps"))),
            "log.txt": open(os.path.join(d, "log.txt")).read(),
            "dtime.txt": open(os.path.join(d, "dtime.txt")).read(),
        }

    cfg = small(n_steps=40)
    st = three(cfg)
    for name, a in zip(FIELDS, (st[1], st[2], st[3], st[0])):
        out[f"three_init_{name}"] = a
    record("fixed40", cfg, st)
    relax_cfg = small(n_steps=300, x_equilibrium=0.0)
    relaxed = solver.run(relax_cfg, *cp(st), out_dir=os.path.join(tmp, "relax"), verbose=False)
    relaxed = (relaxed.eta, relaxed.X, relaxed.X_al, relaxed.X_th)
    for name, a in zip(("eta", "X", "X_al", "X_th"), relaxed):
        out[f"relaxed_{name}"] = a
    record("accepted30", small(n_steps=30, x_equilibrium=0.2), relaxed)
    record("enlarged40", small(n_steps=40, x_equilibrium=0.2, dtime_s=60, dtime_max=150, residual_min=7.6e-4),
           relaxed)
    record("rejected40", small(n_steps=40, x_equilibrium=0.2), st)
    np.savez_compressed(os.path.join(HERE, "reference_small.npz"), **out)
    with open(os.path.join(HERE, "reference_small_logs.json"), "w") as f:
        json.dump(logs, f, indent=1)

    # archived 2022 run
    arch = {}
    m = np.load(os.path.join(ref, "data", "reference", "reproducible_run", "map0.07s_400_400.00K.npz"))
    summarize("map_", {k: m[k] for k in FIELDS}, arch)
    for k in m.files:
        if k not in FIELDS:
            arch[f"mapkey_{k}"] = m[k]
    arch["map_files"] = np.array(m.files)
    line = open(os.path.join(ref, "data", "reference", "reproducible_run", "dtime.txt")).read().splitlines()[1]
    arch["dtime_line1"] = np.array(line.rstrip())
    h = np.load(os.path.join(ref, "data", "histories", "reproducible_run.npz"))
    for k in ("time_out", "T_out", "surf_out", "X_al_mean_out", "X_th_mean_out", "eta_mean_out"):
        arch[f"hist20_{k}"] = h[k][:20]
    np.savez_compressed(os.path.join(HERE, "archived_735.npz"), **arch)

    # 160^2 synthetic microstructure, 20 steps
    cfg_g, spec = workloads.demo160(n_steps=20)
    state = workloads.initial_state(cfg_g, spec)
    rcfg = SimulationConfig(**{k: v for k, v in cfg_g.to_dict().items()})
    rcfg.material_tables = tables
    res = solver.run(rcfg, *cp(state), out_dir=os.path.join(tmp, "demo160"), verbose=False)
    demo = {}
    summarize("init_", dict(zip(("eta", "X", "X_al", "X_th"), state)), demo)
    summarize("final_", {k: getattr(res, k) for k in FIELDS}, demo)
    for name in HISTORIES:
        demo[f"h_{name}"] = np.asarray(res.history[name], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "reference_demo160.npz"), **demo)
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    _ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PF_KKS_REFERENCE")
    if not _ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_CHECKOUT (or set PF_KKS_REFERENCE)")
    main(_ref)
