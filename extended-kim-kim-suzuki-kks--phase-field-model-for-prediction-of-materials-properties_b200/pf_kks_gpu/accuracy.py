"""Accuracy of the mixed-precision step against the all-FP64 step.

Both precisions run the same workload from the same initial state through the
public ``solver.run``. With the adaptive scheme armed, a residual that lands on
the accept / reject threshold can be decided differently by the two
precisions, after which the runs follow different (equally admissible) dt
sequences; ``--fixed-dt`` keeps the scheme unarmed so that both share one time
axis. The report gives the relative L2 error of the final
eta, X, X_al and X_th and, for every history scalar (matrix Si, precipitate
fraction, interface measure, temperature, time, ...), the largest deviation
relative to the scalar's range over the run. Both histories are also written
as ``.npz`` files with the map keys of the reference (``T_out``,
``time_out``, ``eta_mean_out``, ``X_al_mean_out``, ``X_th_mean_out``,
``surf_out``), which is the input of the reference's simulated DSC
(``pf_kks/postprocess/dsc.py:78-130``).

    python -m pf_kks_gpu.accuracy --workload ramp1420 --steps 6000 --fixed-dt --out DIR
"""

import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import solver, workloads

MAP_KEYS = {"time": "time_out", "T": "T_out", "X_al_mean": "X_al_mean_out", "X_th_mean": "X_th_mean_out",
            "eta_mean": "eta_mean_out", "surf": "surf_out"}


def _rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def history_deviation(test, ref):
    """Largest deviation of a history series from the reference series, in
    absolute terms and relative to the reference's range. Entries that are
    NaN in either run (means over empty masks, as in the reference) are left
    out and counted when only one run has them."""
    ha = np.asarray(test, dtype=np.float64)
    hb = np.asarray(ref, dtype=np.float64)
    if ha.shape != hb.shape or hb.size == 0:
        return {"shape_test": list(ha.shape), "shape_ref": list(hb.shape)}
    nan_a, nan_b = np.isnan(ha), np.isnan(hb)
    ok = ~(nan_a | nan_b)
    entry = {"nan_mismatch": int(np.count_nonzero(nan_a != nan_b))}
    if np.any(ok):
        span = float(np.max(hb[ok]) - np.min(hb[ok]))
        scale = span if span > 0 else max(float(np.max(np.abs(hb[ok]))), 1e-300)
        dev = float(np.max(np.abs(ha[ok] - hb[ok])))
        entry.update(max_abs_dev=dev, max_dev_over_range=dev / scale)
    return entry


def run_precision(cfg, state, precision, device=0):
    """One run through solver.run; returns (result, wall seconds)."""
    with tempfile.TemporaryDirectory() as tmp:
        t0 = time.perf_counter()
        res = solver.run(cfg, *state, out_dir=tmp, write_logs=False, verbose=False, precision=precision,
                         device=device)
        wall = time.perf_counter() - t0
    return res, wall


def compare(cfg, state, device=0, out_dir=None, tag="run"):
    """Run mixed and FP64 from the same state; return the report dict."""
    res = {}
    walls = {}
    for prec in ("fp64", "mixed"):
        res[prec], walls[prec] = run_precision(cfg, state, prec, device)
    a, b = res["mixed"], res["fp64"]
    report = {
        "grid": [cfg.nx, cfg.ny],
        "steps": len(b.history["T"]),
        "T_end_K": float(np.asarray(b.history["T"])[-1]),
        "wall_s": walls,
        "good_step": {"fp64": b.good_step, "mixed": a.good_step},
        "fields_rel_l2": {name: _rel_l2(getattr(a, name), getattr(b, name)) for name in ("eta", "X", "X_al", "X_th")},
        "histories": {},
    }
    for name in solver.HIST_NAMES:
        report["histories"][name] = history_deviation(a.history[name], b.history[name])
    if out_dir:
        os.makedirs(out_dir, exist_ok=True)
        for prec, r in res.items():
            arrays = {MAP_KEYS.get(k, k): np.asarray(v) for k, v in r.history.items() if k in solver.HIST_NAMES}
            np.savez_compressed(os.path.join(out_dir, f"{tag}_history_{prec}.npz"), **arrays)
        with open(os.path.join(out_dir, f"{tag}_accuracy.json"), "w") as f:
            json.dump(report, f, indent=1)
    return report


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", default="ramp1420", choices=("ramp1420", "demo160", "iso735"))
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=None, help="directory for the histories and the JSON report")
    ap.add_argument("--fixed-dt", action="store_true",
                    help="x_equilibrium = 0: the adaptive scheme never arms, both precisions share one time axis")
    args = ap.parse_args(argv)
    cfg, spec = getattr(workloads, args.workload)(n_steps=args.steps, seed=args.seed)
    if args.fixed_dt:
        cfg.x_equilibrium = 0.0
    state = workloads.initial_state(cfg, spec)
    tag = args.workload + ("_fixed" if args.fixed_dt else "")
    report = compare(cfg, state, device=args.device, out_dir=args.out, tag=tag)
    print(json.dumps(report, indent=1))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
