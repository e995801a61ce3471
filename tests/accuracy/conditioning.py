"""Record: how the heating workloads amplify small perturbations of the state.

    python tests/accuracy/conditioning.py [--workload demo160] [--steps 6000] [--out FILE]

The mixed step's field errors against the FP64 step grow through the
precipitation stage (about 4e-6 after 6000 fixed-dt steps of demo160 and
ramp1420, from ~1e-7 in the first 3000 steps). This record measures, with the
oracle alone (CPU, FP64), how much the workload itself amplifies a small
perturbation of its state, at fixed dt (x_equilibrium = 0: the adaptive scheme
never arms, so every run shares one time axis):

* ``perturbed``: the run from an initial eta perturbed by seeded Gaussian
  noise of relative size 1e-10 (far above FP64 round-off, far below any
  non-linear effect); its distance from the unperturbed run divided by 1e-10
  is the amplification of a state perturbation up to that step.
* ``perturbed_fp32``: the same with relative size 6e-8 (the FP32 unit
  round-off) on eta and X, once, at the start: the error that a single FP32
  rounding of the state would leave after that many steps.

* ``mixed``: the oracle with the mixed CUDA step's increment form emulated in
  single precision (every transform FP32, increments added to the FP64 state;
  ``oracle.kks_oracle._mixed_update``): the error of FP32 transforms alone.
* ``mixed_ch64``: the same with the Cahn-Hilliard chain (eta gradients, flux
  transforms, FT(X), d_X^) in FP64: how much of that error the
  Cahn-Hilliard transforms carry.

Relative L2 distances of eta and X from the unperturbed FP64 run are recorded
at snapshot steps. Writes a JSON record (committed beside this script).
"""

import argparse
import json
import multiprocessing as mp
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import conftest  # noqa: E402,F401  (puts the package and the oracle on sys.path)

PERTURBATION = 1e-10
FP32_ROUNDOFF = 2.0**-24
VARIANTS = ("fp64", "perturbed", "perturbed_fp32", "mixed", "mixed_ch64")


def _run(job):
    """One oracle run; returns the (eta, X) snapshots by step."""
    name, workload, steps, snap = job
    from oracle import kks_oracle
    from pf_kks_gpu import workloads

    cfg, spec = getattr(workloads, workload)(n_steps=steps)
    cfg.x_equilibrium = 0.0
    eta, X, X_al, X_th = (np.array(a, dtype=np.float64) for a in workloads.initial_state(cfg, spec))
    rng = np.random.default_rng(12345)
    if name == "perturbed":
        eta = eta + PERTURBATION * np.sqrt(np.mean(eta**2)) * rng.standard_normal(eta.shape)
    if name == "perturbed_fp32":
        eta = eta + FP32_ROUNDOFF * np.sqrt(np.mean(eta**2)) * rng.standard_normal(eta.shape)
        X = X + FP32_ROUNDOFF * np.sqrt(np.mean(X**2)) * rng.standard_normal(X.shape)
    update = name if name in ("mixed", "mixed_ch64") else "fp64"
    t0 = time.perf_counter()
    with tempfile.TemporaryDirectory() as d:
        res = kks_oracle.run(cfg, eta, X, X_al, X_th, cfg.material_tables, out_dir=d, write_logs=False,
                             save_maps=False, snapshot_steps=tuple(snap), update=update)
    out = {s: (np.array(v["state"][0]), np.array(v["state"][1])) for s, v in res.snapshots.items()}
    out[steps] = (np.array(res.eta), np.array(res.X))
    T = {s: float(res.history["T"][s - 1]) for s in out if s >= 1}
    return name, out, T, time.perf_counter() - t0


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="demo160")
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--every", type=int, default=500)
    ap.add_argument("--out", default=os.path.join(HERE, "conditioning.json"))
    args = ap.parse_args(argv)
    snap = list(range(args.every, args.steps, args.every))
    jobs = [(n, args.workload, args.steps, snap) for n in VARIANTS]
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        results = {name: (out, T, sec) for name, out, T, sec in pool.map(_run, jobs)}
    base, T, _ = results["fp64"]
    record = {"workload": args.workload, "steps": args.steps, "fixed_dt": True, "perturbation": PERTURBATION,
              "perturbation_fp32": FP32_ROUNDOFF,
              "seconds": {k: v[2] for k, v in results.items()}, "rows": []}
    for s in sorted(base):
        row = {"step": s, "T": T.get(s)}
        for name in VARIANTS[1:]:
            e, x = results[name][0][s]
            row[f"{name}_eta"] = _rel(e, base[s][0])
            row[f"{name}_X"] = _rel(x, base[s][1])
        row["amplification_eta"] = row["perturbed_eta"] / PERTURBATION
        record["rows"].append(row)
    with open(args.out, "w") as f:
        json.dump(record, f, indent=1)
    for row in record["rows"]:
        print(json.dumps(row))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
