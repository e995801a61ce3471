"""Record: the benchmark's first two configurations run in full against the oracle.

    python tests/accuracy/configs_1_2.py [--out tests/accuracy/configs_1_2.json]

* Config 1 (demo160: 160^2, 4 Voronoi cells, ~40 particles, 400 -> 850 K at
  20 K/min, 2000 adaptive steps, FP64): the FP64 GPU step and the oracle from
  the same initial state; relative L2 of the four fields, the largest relative
  deviation of every history, the adaptive decisions, and the mixed step's
  errors beside them.
* Config 2 (iso735: 735^2, 20 cells, ~300 particles, isothermal 500 K, 500
  fixed-dt steps): the oracle (reference CPU FP64), the FP64 GPU step and the
  mixed GPU step; relative L2 of eta and X and the error of the matrix Si mean,
  the precipitate fraction (mean eta) and the interface measure, at the end and
  as the largest deviation over the run, each GPU precision against the oracle.

Needs a GPU; the oracle uses every host core for its FFTs. Writes a JSON record
(committed beside this script).
"""

import argparse
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import conftest  # noqa: E402,F401  (puts the package and the oracle on sys.path)

FIELDS = ("eta", "X", "X_al", "X_th")
SCALARS = {"matrix_Si_mean": "X_al_mean", "precipitate_fraction": "eta_mean", "interface_measure": "surf"}


def _rel(a, b):
    a, b = np.ravel(np.asarray(a, float)), np.ravel(np.asarray(b, float))
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _hist_dev(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    n = min(a.size, b.size)  # runs whose adaptive decisions differ keep histories of different lengths
    a, b = a[:n], b[:n]
    ok = ~(np.isnan(a) | np.isnan(b))
    if not np.any(ok):
        return None
    scale = max(float(np.max(np.abs(b[ok]))), 1e-300)
    return float(np.max(np.abs(a[ok] - b[ok])) / scale)


def _decisions(log_path):
    out = []
    with open(log_path) as f:
        for line in f:
            if ": RE>resmax" in line:
                out.append((int(line.split()[1].rstrip(":")), "rejected"))
            elif "(resmin <RE <resmax)" in line:
                out.append((int(line.split()[1].rstrip(",")), "accepted"))
            elif ":RE <resmin" in line:
                out.append((int(line.split()[-1]), "enlarged"))
    return out


def _gpu(cfg, state, precision, out_dir):
    from pf_kks_gpu import solver

    t0 = time.time()
    res = solver.run(cfg, *[np.array(a, copy=True) for a in state], out_dir=out_dir, verbose=False,
                     precision=precision)
    return res, time.time() - t0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "configs_1_2.json"))
    args = ap.parse_args(argv)
    from oracle import kks_oracle
    from pf_kks_gpu import workloads

    rec = {}
    tmp = tempfile.mkdtemp()
    workers = os.cpu_count()

    cfg, spec = workloads.demo160(n_steps=2000)
    state = workloads.initial_state(cfg, spec)
    t0 = time.time()
    ref = kks_oracle.run(cfg, *[np.array(a, copy=True) for a in state], cfg.material_tables,
                         out_dir=os.path.join(tmp, "c1_cpu"), fft_workers=workers)
    t_ref = time.time() - t0
    f64, t64 = _gpu(cfg, state, "fp64", os.path.join(tmp, "c1_fp64"))
    mix, tmx = _gpu(cfg, state, "mixed", os.path.join(tmp, "c1_mixed"))
    dref = _decisions(os.path.join(tmp, "c1_cpu", "log.txt"))
    rec["config1_demo160"] = {
        "steps": len(ref.history["T"]), "T_end_K": float(ref.history["T"][-1]),
        "good_step": {"oracle": ref.good_step, "fp64": f64.good_step, "mixed": mix.good_step},
        "adaptive_decisions": {"oracle": len(dref),
                               "fp64_same": _decisions(os.path.join(tmp, "c1_fp64", "log.txt")) == dref,
                               "mixed_same": _decisions(os.path.join(tmp, "c1_mixed", "log.txt")) == dref},
        "logs_identical_fp64": all(open(os.path.join(tmp, "c1_fp64", n)).read()
                                   == open(os.path.join(tmp, "c1_cpu", n)).read() for n in ("log.txt", "dtime.txt")),
        "fields_rel_l2": {"fp64": {n: _rel(getattr(f64, n), getattr(ref, n)) for n in FIELDS},
                          "mixed": {n: _rel(getattr(mix, n), getattr(ref, n)) for n in FIELDS}},
        "history_max_rel_dev": {"fp64": {k: _hist_dev(f64.history[k], ref.history[k]) for k in ref.history},
                                "mixed": {k: _hist_dev(mix.history[k], ref.history[k]) for k in SCALARS.values()}},
        "wall_s": {"oracle": t_ref, "fp64": t64, "mixed": tmx, "oracle_fft_workers": workers},
    }
    print("config1", {k: v for k, v in rec["config1_demo160"].items() if k != "history_max_rel_dev"}, flush=True)

    cfg, spec = workloads.iso735(n_steps=500)
    state = workloads.initial_state(cfg, spec)
    t0 = time.time()
    ref = kks_oracle.run(cfg, *[np.array(a, copy=True) for a in state], cfg.material_tables,
                         out_dir=os.path.join(tmp, "c2_cpu"), fft_workers=workers)
    t_ref = time.time() - t0
    f64, t64 = _gpu(cfg, state, "fp64", os.path.join(tmp, "c2_fp64"))
    mix, tmx = _gpu(cfg, state, "mixed", os.path.join(tmp, "c2_mixed"))
    entry = {"steps": len(ref.history["T"]), "wall_s": {"oracle": t_ref, "fp64": t64, "mixed": tmx,
                                                        "oracle_fft_workers": workers}}
    for name, res in (("fp64", f64), ("mixed", mix)):
        e = {"eta_rel_l2": _rel(res.eta, ref.eta), "X_rel_l2": _rel(res.X, ref.X)}
        for label, key in SCALARS.items():
            a, b = np.asarray(res.history[key], float), np.asarray(ref.history[key], float)
            e[label] = {"oracle_end": float(b[-1]), "gpu_end": float(a[-1]),
                        "rel_error_end": abs(float(a[-1] - b[-1])) / max(abs(float(b[-1])), 1e-300),
                        "max_rel_dev_over_run": _hist_dev(a, b)}
        entry[name] = e
    rec["config2_iso735"] = entry
    print("config2", json.dumps(entry)[:1500], flush=True)
    with open(args.out, "w") as f:
        json.dump(rec, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
