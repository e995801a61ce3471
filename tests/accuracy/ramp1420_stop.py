"""Record: where the 1420^2 heating run (ramp1420, adaptive dt) stops, and
whether the oracle stops there too.

    python tests/accuracy/ramp1420_stop.py [--back 12] [--out tests/accuracy/ramp1420_stop.json]

1. The FP64 GPU step runs ramp1420 from its initial state until the adaptive
   scheme stops the run (AdaptiveStepError: no admissible dt after
   max_iterations attempts, pf_kks/solver.py:292-295) or 6000 steps pass.
2. A second FP64 cell runs the same steps up to ``back`` steps before the
   stop, and no later than the step at which the adaptive scheme arms (the run
   is deterministic: the same kernels give the same bits), and hands its
   complete loop state to the oracle (fields, scalars and history rows;
   tests/conftest.py:gpu_loop_state), which then arms by itself.
3. The oracle (FP64 numpy, every host core for its FFTs) continues from there
   and the adaptive decisions of both, attempt by attempt, are compared, with
   the residual each attempt computed.
4. The mixed step runs the same workload to its own stop; its decisions are
   compared with the FP64 step's.

Needs a GPU. Writes a JSON record (committed beside this script).
"""

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
sys.path.insert(0, TESTS)

import conftest  # noqa: E402,F401  (puts the package and the oracle on sys.path)
from conftest import gpu_loop_state  # noqa: E402

MAX_STEPS = 6000


def _gpu_run(cfg, state, tables, precision, n_steps, chunk=500):
    """Run a fresh cell up to n_steps or its stop; (cell, status, decisions, rows)."""
    from pf_kks_gpu import _lib as L
    from pf_kks_gpu import solver

    kinds = {L.KKS_REC_REJECTED: "rejected", L.KKS_REC_ACCEPTED: "accepted", L.KKS_REC_ENLARGED: "enlarged"}
    cell = solver.Cell(cfg, tables, precision=precision)
    cell.upload(*state)
    decisions, rows = [], []
    status = 0
    while cell.state().istep < n_steps:
        status = cell.run(min(chunk, n_steps - cell.state().istep))
        recs, r = cell.drain()
        decisions += [(int(x.istep), kinds[x.kind], float(x.res_total),
                       {"energy_derivative": x.res_energy_derivative, "diffusion": x.res_diffusion,
                        "allen_cahn": x.res_allen_cahn, "temperature": x.res_temperature, "dtime_s": x.dtime_s})
                      for x in recs if x.kind in kinds]
        rows.append(r)
        if status != 0:
            break
    return cell, status, decisions, np.concatenate(rows)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--back", type=int, default=12, help="steps before the stop at which the oracle takes over")
    ap.add_argument("--out", default=os.path.join(HERE, "ramp1420_stop.json"))
    args = ap.parse_args(argv)

    from oracle import kks_oracle
    from pf_kks_gpu import _lib as L
    from pf_kks_gpu import workloads
    from pf_kks_gpu.materials import MaterialTables

    cfg, spec = workloads.ramp1420(n_steps=MAX_STEPS, precision="fp64")
    state = workloads.initial_state(cfg, spec)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    rec = {"workload": "ramp1420: 1420^2, 40 Voronoi cells, ~1200 particles, 400->719 K at 20 K/min, adaptive dt",
           "max_steps": MAX_STEPS}

    t0 = time.time()
    cell, status, dec64, rows64 = _gpu_run(cfg, state, tables, "fp64", MAX_STEPS)
    s = cell.state()
    cell.close()
    stop = int(s.error_istep) if status else None
    rec["fp64"] = {"status": int(status), "steps_done": int(s.istep), "stop_step": stop,
                   "good_step": int(s.good_step) if s.flag else None, "attempts": int(s.attempts),
                   "T_at_end_K": float(rows64[-1, L.H["T"]]),
                   "X_al_mean_at_end": float(rows64[-1, L.H["X_al_mean"]]), "wall_s": time.time() - t0,
                   "decisions": len(dec64), "rejections": sum(d[1] == "rejected" for d in dec64),
                   "first_decisions": dec64[:3], "last_decisions": dec64[-3:]}
    print("fp64", rec["fp64"], flush=True)

    if stop is not None:
        # before the scheme arms (flag is set at the end of step good_step), so that the
        # oracle arms by itself; the state then carries no residual pair
        start = max(min(stop - args.back, int(s.good_step) if s.flag else stop - args.back), 1)
        cell, st, _, rows = _gpu_run(cfg, state, tables, "fp64", start)
        assert st == 0 and cell.state().istep == start
        resume, fields = gpu_loop_state(cell, rows)
        cell.close()
        seen = []
        t0 = time.time()
        err = None
        try:
            kks_oracle.run(cfg, *fields, cfg.material_tables, write_logs=False, save_maps=False,
                           fft_workers=os.cpu_count(), resume=resume, on_attempt=seen.append, max_steps=stop + 2)
        except kks_oracle.AdaptiveStepError as exc:
            err = str(exc)
        gpu_tail = [d for d in dec64 if d[0] >= start]
        ora = [(a["istep"], a["decision"], float(a["residual"].total)) for a in seen if a["decision"] != "none"]
        same = [g[:2] for g in gpu_tail] == [o[:2] for o in ora]
        rel = [abs(g[2] - o[2]) / max(abs(o[2]), 1e-300) for g, o in zip(gpu_tail, ora)]
        msg = (f"step {s.error_istep}: no admissible time step after {s.error_iteration} attempts "
               f"(dtime_s={s.error_dtime_s:.2e})")
        rec["oracle_from_gpu_state"] = {
            "start_step": start, "oracle_error": err, "gpu_error": msg, "same_error": err == msg,
            "decisions_compared": len(ora), "same_decisions": same,
            "max_rel_residual_diff": max(rel) if rel else None,
            "residuals_first": [(g[0], g[1], g[2], o[2]) for g, o in list(zip(gpu_tail, ora))[:8]],
            "residuals_last": [(g[0], g[1], g[2], o[2]) for g, o in list(zip(gpu_tail, ora))[-4:]],
            "wall_s": time.time() - t0}
        print("oracle", {k: v for k, v in rec["oracle_from_gpu_state"].items() if not k.startswith("resid")},
              flush=True)

    t0 = time.time()
    cfgm, _ = workloads.ramp1420(n_steps=MAX_STEPS, precision="mixed")
    cell, status_m, decm, rowsm = _gpu_run(cfgm, state, tables, "mixed", MAX_STEPS)
    sm = cell.state()
    cell.close()
    first_diff = next((k for k, (a, b) in enumerate(zip(decm, dec64)) if a[:2] != b[:2]), None)
    rec["mixed"] = {"status": int(status_m), "steps_done": int(sm.istep),
                    "stop_step": int(sm.error_istep) if status_m else None,
                    "good_step": int(sm.good_step) if sm.flag else None, "attempts": int(sm.attempts),
                    "decisions": len(decm), "same_decisions_as_fp64": first_diff is None and len(decm) == len(dec64),
                    "first_different_decision": None if first_diff is None else
                    {"mixed": decm[first_diff], "fp64": dec64[first_diff] if first_diff < len(dec64) else None},
                    "wall_s": time.time() - t0}
    print("mixed", rec["mixed"], flush=True)
    with open(args.out, "w") as f:
        json.dump(rec, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
