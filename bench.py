"""Benchmark: KKS steps/s of the semi-implicit step at 1420^2 on B200.

Workload (the reference-metric configuration that fits one GPU): the 1420 x 1420
cell (710 nm, 40 Voronoi cells, ~1200 particles of radius U(3,10), heated
400 -> 719 K at 20 K/min, energy-residual adaptive dt), mixed FP32/FP64 step.
One step = one attempt of the time loop over the whole cell; the inputs (4
fields of 1420^2) are resident in HBM when the timed region starts, and the
per-attempt working set (~300 MB) is larger than the 126 MB L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank advances its own cell
(seed = rank): the ensemble shards with no collective in the step, so the
scaling is weak; the device time is the max over ranks.

``--impl reference`` times the CPU oracle (a numpy restatement of the
reference's ``pf_kks.solver.run`` step, run with every host core for its FFTs)
on the same workload, rank 0 only.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "extended-kim-kim-suzuki-kks--phase-field-model-for-prediction-of-materials-properties_b200")
for _p in (PKG, REPO):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "KKS steps/s @1420^2 (mixed FP32/FP64 step)"
UNIT = "steps/s"
# Algorithmic HBM traffic of one attempt in units of one N-element real field
# (every array touched once; 2-D transforms counted as a single pass):
# state 8 + forward spectra 12 + C2R outputs 10 + pre-inverse spectra 4 +
# non-state R2C inputs 8 = 42; armed steps add the residual pair (7) = 49.
UNITS_UNARMED = 42
UNITS_ARMED = 49


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 7:
                    continue
                try:
                    sm.append(float(parts[0]))
                    mx.append(float(parts[1]))
                except ValueError:
                    continue
                for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                   parts[3:7]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def bench_config(armed):
    """The workload of both arms (the same keys and values for the GPU line and
    the reference line; precision, attempts and launch shape are top-level
    keys of each line)."""
    return {
        "workload": "ramp1420: 1420x1420 KKS cell (710 nm), 40 Voronoi cells, ~1200 particles R~U(3,10), "
                    "400->719 K at 20 K/min, adaptive dt; one cell per GPU",
        "grid": [1420, 1420],
        "armed": bool(armed),
        "l2": "inputs larger than L2: an unarmed attempt touches ~160 MB (FP64 state in and out 96 MB, spectra 64 MB) > 126 MB L2; no flush",
    }


def make_workload(precision, seed):
    from pf_kks_gpu import workloads

    cfg, spec = workloads.ramp1420(n_steps=100000, precision=precision, seed=seed)
    return cfg, spec, workloads.initial_state(cfg, spec)


def run_reference(args):
    """CPU arm: the oracle's step on the same workload, every host core for the
    FFTs. The first steps of the workload are unarmed (the adaptive scheme arms
    once the matrix Si mean falls to x_equilibrium), as in the GPU arm's timed
    steps. W warm-up steps, then K timed steps, each capped so that the arm
    ends within a few minutes."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    from oracle import kks_oracle

    cores = os.cpu_count() or 1
    cfg, spec, state = make_workload("fp64", 0)
    budget_s = 150.0
    warm = args.warmup
    t0 = time.perf_counter()
    kks_oracle.run(cfg, *state, cfg.material_tables, write_logs=False, save_maps=False, max_steps=warm,
                   fft_workers=cores)
    per_step = (time.perf_counter() - t0) / max(warm, 1)
    k = max(1, min(args.steps, int(budget_s / max(per_step, 1e-3))))
    t0 = time.perf_counter()
    res = kks_oracle.run(cfg, *state, cfg.material_tables, write_logs=False, save_maps=False, max_steps=k,
                         fft_workers=cores)
    dt = time.perf_counter() - t0
    value = k / dt
    sample = (f"{k} steps of the 1420^2 workload from its initial state (FP64 numpy oracle, scipy.fft with {cores} "
              f"workers; its elasticity is the closed 2-D form, so it is faster than the reference's own einsum "
              f"elasticity, ~10 s/step at 1420^2)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": k,
        "warmup": warm, "ms_per_step": 1000.0 * dt / k, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(armed=False),
        "precision": "fp64", "attempts": int(res.attempts),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline(state, cfg):
    """Bounded CPU sample of the same workload for the GPU arm's line."""
    from oracle import kks_oracle

    cores = os.cpu_count() or 1
    k = 3
    t0 = time.perf_counter()
    kks_oracle.run(cfg, *state, cfg.material_tables, write_logs=False, save_maps=False, max_steps=k,
                   fft_workers=cores)
    dt = time.perf_counter() - t0
    return {"value": k / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first {k} steps of the same 1420^2 cell, FP64 numpy oracle, scipy.fft with {cores} workers"}


def _oracle_cell_steps(job):
    """One CPU process of the ensemble baseline: ``k`` FP64 oracle steps of one
    cell (numpy, one FFT worker); returns (cell-steps, seconds of the steps)."""
    from oracle import kks_oracle

    cfg, state, k = job
    t0 = time.perf_counter()
    kks_oracle.run(cfg, *state, cfg.material_tables, write_logs=False, save_maps=False, max_steps=k,
                   fft_workers=1)
    return cfg.nx * cfg.ny * k, time.perf_counter() - t0


def ensemble_cpu_baseline(members, k=3):
    """The ensemble on the host cores: one independent oracle process per core,
    each advancing one cell of the ensemble by ``k`` steps (the first ``cores``
    cells); throughput = all cell-steps / the longest process's step time.
    Processes are started with ``spawn`` (this process has a CUDA context)."""
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    jobs = [(cfg, state, k) for cfg, state in members[:cores]]
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        out = pool.map(_oracle_cell_steps, jobs)
    work = sum(w for w, _ in out)
    return {"value": work / max(t for _, t in out), "unit": "cell-steps/s", "cores": len(jobs), "kind": "port",
            "sample": f"{len(jobs)} concurrent processes (one per core), each {k} FP64 oracle steps of one "
                      f"ensemble cell (sides {sorted({c.nx for c, _, _ in jobs})}), numpy with one FFT worker"}


def ensemble_leg(precision, device, steps, warmup, cpu=True):
    """Batched cell-steps/s of the 48-cell ensemble (sides 128..512, heating
    rates U(5,40) K/min): the batch (kks_batch_run: every kernel of an attempt
    launched once for all cells, one graph per batch attempt), every cell on
    its own stream (kks_run_many) and one cell after the other;
    ``cell_steps_per_s`` is the faster of the first two (the mode the tuned
    ensemble runs in)."""
    from pf_kks_gpu import workloads
    from pf_kks_gpu.ensemble import Ensemble

    members = [(cfg, workloads.initial_state(cfg, spec)) for cfg, spec in workloads.ensemble(48, 100000, precision)]
    ens = Ensemble(members, precision=precision, device=device, tune=True)
    try:
        if ens.batch is not None:
            ens.run_batch(warmup)
        ens.run_streams(warmup)

        def advance(fn):
            before = [c.state().istep for c in ens.cells]
            t0 = time.perf_counter()
            fn(steps)
            dt = time.perf_counter() - t0
            done = [c.state().istep - b for c, b in zip(ens.cells, before)]
            return sum(n * d for n, d in zip(ens.points, done)) / dt

        ms0, att0 = ens.batch_timing()
        batched = advance(ens.run_batch) if ens.batch is not None else None
        ms1, att1 = ens.batch_timing()
        streams = advance(ens.run_streams)
        sequential = advance(ens.run_sequential)
    finally:
        ens.close()
    best = max(v for v in (batched, streams) if v is not None)
    out = {"cells": len(members), "points": int(sum(c.nx * c.ny for c, _ in members)), "steps": steps,
           "mode": ens.mode, "mode_ms_per_attempt": ens.mode_ms,
           "launch_shapes": {f"{k[0]}x{k[1]}": v for k, v in sorted(ens.shapes.items())},
           "batch_ms_per_attempt_by_column_tile": ens.batch_tile_ms,
           "batch_ms_per_attempt_by_field_grid_divisor": ens.batch_grid_ms,
           "batch_groups": ens.groups, "batch_ms_per_attempt_by_groups": ens.batch_groups_ms,
           "cell_steps_per_s": best, "batch_cell_steps_per_s": batched, "streams_cell_steps_per_s": streams,
           "sequential_cell_steps_per_s": sequential, "speedup_vs_sequential": best / sequential,
           "timing": "host wall clock around each run call (one host sync per batch of attempts)"}
    if att1 > att0:
        out["batch_device_ms_per_attempt"] = (ms1 - ms0) / (att1 - att0)
    if cpu:
        out["cpu_baseline"] = ensemble_cpu_baseline(members)
    return out


def armed_leg(precision, device, tables, peak, max_attempts=49):
    """Armed attempts of the 1420^2 heating run: the adaptive scheme arms at
    step 3638 and from step 3640 every attempt computes the energy residual
    (the residual pair adds 7 N-arrays: 49 units per attempt). The run is
    advanced to step 3640 untimed; then one kks_run(1) takes the attempts of
    that step (all rejected, the reference's behaviour on this workload, until
    max_iterations stops the run) and their device time is measured."""
    from pf_kks_gpu import solver, workloads

    cfg, spec = workloads.ramp1420(n_steps=3700, precision=precision)
    cell = solver.Cell(cfg, tables, precision=precision, device=device)
    try:
        cell.upload(*workloads.initial_state(cfg, spec))
        cell.run(3640)
        cell.drain()
        s = cell.state()
        m0, a0 = cell.timing()
        cell.run(1)
        m1, a1 = cell.timing()
        s1 = cell.state()
        cell.drain()
    finally:
        cell.close()
    att = int(s1.attempts - s.attempts)
    ms = (m1 - m0) / max(att, 1)
    N = cfg.nx * cfg.ny
    p = 8 if precision == "fp64" else 4
    achieved = UNITS_ARMED * N * p / (ms / 1000.0) / 1e9
    return {"step": int(s.istep), "good_step": int(s.good_step), "armed": bool(s.flag), "attempts": att,
            "status": int(s1.status), "ms_per_attempt": ms, "units": UNITS_ARMED,
            "algorithmic_bytes": UNITS_ARMED * N * p, "achieved_gbs": achieved, "frac": achieved / peak,
            "timing": "CUDA events around kks_run on the cell's stream; the attempts of step 3640"}


def sharded_ensemble_leg(precision, device, steps, warmup, rank, world, barrier, max_over_ranks):
    """The 48-cell ensemble sharded over the job's ranks (one GPU each): every
    rank builds and advances only its cost-balanced shard
    (pf_kks_gpu.ensemble.partition) as one tuned Ensemble; no collective in the
    steps. Whole-job cell-steps/s = all cells' points x steps / the slowest
    rank's wall time."""
    import torch

    from pf_kks_gpu import workloads
    from pf_kks_gpu.ensemble import Ensemble, cell_cost, partition

    specs = workloads.ensemble(48, 100000, precision)
    shard = partition([cell_cost(c.nx, c.ny, steps) for c, _ in specs], world)[rank]
    members = [(specs[i][0], workloads.initial_state(*specs[i])) for i in shard]
    ens = Ensemble(members, precision=precision, device=device, tune=True) if members else None
    try:
        if ens is not None:
            ens.run(warmup)
        barrier()
        t0 = time.perf_counter()
        if ens is not None:
            ens.run(steps)
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t0)
    finally:
        if ens is not None:
            ens.close()
    points = sum(c.nx * c.ny for c, _ in specs)
    return {"cells": len(specs), "points": int(points), "steps": steps, "ranks": world,
            "cells_on_rank0": len(shard) if rank == 0 else None, "cell_steps_per_s": points * steps / dt,
            "timing": "host wall clock per rank around Ensemble.run, max over ranks"}


def profile_armed(args):
    """Profiling run of armed attempts at 1420^2 that a kernel profiler can
    reach in few launches. ``save`` advances the ramp1420 cell untimed to step
    3640 (the adaptive scheme is armed from step 3638) and writes its
    checkpoint to ``--checkpoint``. ``measure`` runs 3 unarmed attempts of a
    fresh cell (30 kernels), then restores the checkpoint into a second cell
    and runs step 3640 (its attempts are all rejected until max_iterations
    stops the run: every attempt computes the residual pair and restores the
    step's input), printing both cells' device ms per attempt."""
    from pf_kks_gpu import solver, workloads
    from pf_kks_gpu.materials import MaterialTables

    cfg, spec = workloads.ramp1420(n_steps=3700, precision=args.precision)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    shape = [int(v) for v in (args.shape or "1,3,296").split(",")]
    init = workloads.initial_state(cfg, spec)
    if args.armed_profile == "save":
        cell = solver.Cell(cfg, tables, precision=args.precision)
        try:
            cell.set_launch_shape(*shape)
            cell.upload(*init)
            cell.run(3640)
            cell.drain()
            with open(args.checkpoint, "wb") as f:
                f.write(cell.checkpoint())
            print(json.dumps({"saved": args.checkpoint, "istep": int(cell.state().istep)}), flush=True)
        finally:
            cell.close()
        return 0
    out = {}
    a = solver.Cell(cfg, tables, precision=args.precision)
    try:
        a.set_launch_shape(*shape)
        a.upload(*init)
        m0, n0 = a.timing()
        a.run(3)
        m1, n1 = a.timing()
        out["unarmed_ms_per_attempt"] = (m1 - m0) / max(n1 - n0, 1)
    finally:
        a.close()
    b = solver.Cell(cfg, tables, precision=args.precision)
    try:
        b.set_launch_shape(*shape)
        with open(args.checkpoint, "rb") as f:
            b.restore(f.read())
        s0 = b.state()
        m0, _ = b.timing()
        b.run(1)
        m1, _ = b.timing()
        s1 = b.state()
        n = int(s1.attempts - s0.attempts)
        out.update({"step": int(s0.istep), "armed": bool(s0.flag), "armed_attempts": n,
                    "armed_ms_per_attempt": (m1 - m0) / max(n, 1), "status": int(s1.status)})
    finally:
        b.close()
    print(json.dumps(out), flush=True)
    return 0


def profile_ensemble(args):
    """Profiling run: the 48-cell ensemble as one batch (column tile 4, one
    group), ``--warmup`` then ``--steps`` batch attempts; device time from the
    batch's CUDA events."""
    from pf_kks_gpu import workloads
    from pf_kks_gpu.ensemble import Ensemble

    members = [(cfg, workloads.initial_state(cfg, spec))
               for cfg, spec in workloads.ensemble(48, 100000, args.precision)]
    ens = Ensemble(members, precision=args.precision, batched=True, cols=4, groups=1)
    try:
        ens.run_batch(args.warmup)
        ms0, a0 = ens.batch_timing()
        ens.run_batch(args.steps)
        ms1, a1 = ens.batch_timing()
        pts = sum(ens.points)
    finally:
        ens.close()
    per = (ms1 - ms0) / max(a1 - a0, 1)
    print(json.dumps({"metric": "batched cell-steps/s (48-cell ensemble, one batch)", "value": pts / (per / 1000.0),
                      "unit": "cell-steps/s", "ms_per_batch_attempt": per, "attempts": int(a1 - a0),
                      "profiling_run": True}), flush=True)
    return 0


def init_leg(precision, device):
    """Initial state of the 1420^2 cell and of the 48-cell ensemble: the host
    generator followed by kks_upload, against the device generator
    (kks_voronoi_edges + kks_generate_fields, the same arrays)."""
    from pf_kks_gpu import solver, workloads
    from pf_kks_gpu.materials import MaterialTables

    out = {}
    for name, members in (("ramp1420", [workloads.ramp1420(n_steps=10, precision=precision)]),
                          ("ensemble48", workloads.ensemble(48, 10, precision))):
        cells = []
        try:
            for cfg, spec in members:
                tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
                cells.append((cfg, spec, solver.Cell(cfg, tables, precision=precision, device=device)))
            workloads.initial_state_on_device(cells[0][2], cells[0][0], cells[0][1])  # first-call set-up
            t0 = time.perf_counter()
            for cfg, spec, cell in cells:
                cell.upload(*workloads.initial_state(cfg, spec))
            host = time.perf_counter() - t0
            t0 = time.perf_counter()
            for cfg, spec, cell in cells:
                workloads.initial_state_on_device(cell, cfg, spec)
            dev = time.perf_counter() - t0
        finally:
            for _, _, cell in cells:
                cell.close()
        out[name] = {"cells": len(members), "points": int(sum(c.nx * c.ny for c, _ in members)),
                     "host_generate_and_upload_s": host, "device_generate_s": dev, "speedup": host / dev}
    out["timing"] = "host wall clock; each call returns after its cell's stream is idle"
    return out


def adjoint_leg(device, steps=300, checkpoint_every=50):
    """adjoint256: the gradient workload. 300 fixed-dt steps at 256^2 through
    the coefficient chain and kks_adj_forward, the simulated DSC of the run,
    the loss against the DSC of the target run (Si mobility x 1.2, vacancy
    annealing rate x 0.8, interface energy x 1.1), and its gradient with
    respect to the log of the three factors through the hand-written adjoint
    (checkpoint every 50 steps, segments recomputed); FP64 and mixed
    precision (FP32 transforms of the increments)."""
    import torch

    from pf_kks_gpu import adjoint as A
    from pf_kks_gpu import workloads
    from pf_kks_gpu.materials import MaterialTables

    cfg, spec = workloads.adjoint256(n_steps=steps)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    state = workloads.initial_state(cfg, spec)
    s0 = A.initial_state_tensor(*state, device=device)
    target = torch.tensor(np.log(workloads.ADJOINT_TARGET_FACTORS), dtype=torch.float64)
    out = {"workload": "adjoint256: 256^2, 8 cells, 500->520 K, 300 fixed-dt steps; loss = squared error of the "
                       "simulated DSC against the run with Si mobility x1.2, annealing rate x0.8, interface "
                       "energy x1.1", "steps": steps, "checkpoint_every": checkpoint_every,
           "timing": "host wall clock, coefficient chain, histories and DSC included"}
    q_target = None
    for precision in ("fp64", "mixed"):
        stepper = A.StepAdjoint.for_config(cfg, tables, device=device, precision=precision)
        if q_target is None:
            with torch.no_grad():
                q_target = A.dsc_of_run(cfg, tables, s0, stepper, steps, target, checkpoint_every).total
        theta = torch.zeros(3, dtype=torch.float64, requires_grad=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        q = A.dsc_of_run(cfg, tables, s0, stepper, steps, theta, checkpoint_every).total
        loss = ((q - q_target) ** 2).sum()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loss.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        stepper.close()
        g = theta.grad.tolist()
        out[precision] = {"loss": float(loss), "forward_s": t1 - t0, "backward_s": t2 - t1,
                          "forward_steps_per_s": steps / (t1 - t0), "gradient_steps_per_s": steps / (t2 - t1),
                          "grad_log_c_D": g[0], "grad_log_anneal_rate": g[1], "grad_log_c_gamma": g[2]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--precision", default="mixed", choices=("mixed", "mixed-cufft", "fp64"))
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shape instead of the autotuner's choice")
    ap.add_argument("--shape", default=None,
                    help="explicit launch shape pipeline,cols,field_blocks (skips the autotuner)")
    ap.add_argument("--only-ensemble", action="store_true",
                    help="profiling: only the 48-cell ensemble as one batch (column tile 4, one group)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 48-cell ensemble leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (gradient) leg")
    ap.add_argument("--no-init", action="store_true", help="skip the initial-state (generator) leg")
    ap.add_argument("--no-armed", action="store_true", help="skip the armed-attempt leg")
    ap.add_argument("--only-timed", action="store_true",
                    help="skip the FP64 comparison and end-to-end cells (profiling runs)")
    ap.add_argument("--armed-profile", default=None, choices=("save", "measure"),
                    help="profiling: armed 1420^2 attempts from a checkpoint at step 3640 (save it, then measure)")
    ap.add_argument("--checkpoint", default=os.path.join(tempfile.gettempdir(), "kks_ramp1420_step3640.bin"),
                    help="checkpoint file of --armed-profile")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.only_ensemble:
        return profile_ensemble(args)
    if args.armed_profile:
        return profile_armed(args)

    rank, world, local_rank = env_rank()
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from pf_kks_gpu import solver
    from pf_kks_gpu.materials import MaterialTables

    cfg, spec, state = make_workload(args.precision, seed=rank)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    N = cfg.nx * cfg.ny
    p = 8 if args.precision == "fp64" else 4

    def barrier():
        if dist is not None:
            import torch

            torch.cuda.synchronize()
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    cell = solver.Cell(cfg, tables, precision=args.precision, device=local_rank)
    cell.upload(*state)
    # launch shape: the autotuner's choice, timed on this cell's own state
    # (restored afterwards), outside the timed region
    tuned = None
    if args.shape:
        cell.set_launch_shape(*[int(v) for v in args.shape.split(",")])
    elif not args.no_autotune and not args.only_timed:
        from pf_kks_gpu import autotune

        tuned = autotune.tune(cell, attempts=20, device=local_rank, cache=False)
    shape = cell.launch_shape()
    fused, kernels_per_attempt = cell.pipeline()
    cell.run(args.warmup)
    cell.drain()
    s0 = cell.state()
    barrier()
    ms0, a0 = cell.timing()
    with ClockSampler(local_rank) as clocks:
        cell.run(args.steps)
    ms1, a1 = cell.timing()
    s1 = cell.state()
    cell.drain()
    barrier()
    dev_ms = max_over_ranks(ms1 - ms0)
    steps_done = s1.istep - s0.istep
    attempts = s1.attempts - s0.attempts
    armed = bool(s1.flag) and s1.istep >= s1.good_step + 2
    value = world * steps_done / (dev_ms / 1000.0)
    ms_per_attempt = (ms1 - ms0) / max(attempts, 1)
    # a longer device timing beside the K timed attempts (launch jitter averages out)
    long_run = None
    if not args.only_timed and args.steps < 200:
        m0, b0 = cell.timing()
        cell.run(200)
        m1, b1 = cell.timing()
        cell.drain()
        long_run = {"attempts": int(b1 - b0), "ms_per_attempt": (m1 - m0) / max(b1 - b0, 1),
                    "steps_per_s": 200 / ((m1 - m0) / 1000.0)}
    cell.close()

    # FP64 step on the same cell, for the mixed-vs-FP64 ratio of the metric
    fp64 = fp64_cufft = fp64_shape = None
    if args.precision != "fp64" and not args.only_timed:
        c64 = solver.Cell(cfg, tables, precision="fp64", device=local_rank)
        c64.upload(*state)
        if not args.no_autotune:
            from pf_kks_gpu import autotune

            autotune.tune(c64, attempts=10, device=local_rank, cache=False)
        c64.run(args.warmup)
        m0, _ = c64.timing()
        k64 = max(10, args.steps // 4)
        c64.run(k64)
        m1, _ = c64.timing()
        fp64 = k64 / ((m1 - m0) / 1000.0)
        fp64_shape = c64.launch_shape()
        c64.close()
        # the same FP64 step with cuFFT transforms (the plain GPU step before the
        # fused FP64 passes), the other denominator of the mixed-vs-FP64 ratio
        c64 = solver.Cell(cfg, tables, precision="fp64", device=local_rank)
        c64.set_launch_shape(0, fp64_shape["cols"], fp64_shape["field_blocks"])
        c64.upload(*state)
        c64.run(args.warmup)
        m0, _ = c64.timing()
        c64.run(k64)
        m1, _ = c64.timing()
        c64.close()
        fp64_cufft = k64 / ((m1 - m0) / 1000.0)

    # end to end through the C ABI: host fields in, K steps, fields and histories out
    import ctypes

    if args.only_timed:
        print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "ms_per_attempt": ms_per_attempt,
                          "attempts": int(attempts), "profiling_run": True}), flush=True)
        return 0

    try:
        import torch

        pinned = [torch.empty(N, dtype=torch.float64).pin_memory().numpy() for _ in range(8)]
    except Exception:
        pinned = [np.empty(N) for _ in range(8)]
    for k in range(4):
        pinned[k][:] = state[k].ravel()
    e2e_cell = solver.Cell(cfg, tables, precision=args.precision, device=local_rank)
    e2e_cell.set_launch_shape(shape["pipeline"], shape["cols"], shape["field_blocks"])
    lib = e2e_cell.lib
    host_in = [pinned[k].ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for k in range(4)]
    host_out = [pinned[4 + k].ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for k in range(4)]
    # warm-up: one whole call (upload, W steps, drain, download into the output buffers)
    lib.kks_upload(e2e_cell.h, *host_in)
    e2e_cell.run(args.warmup)
    e2e_cell.drain()
    lib.kks_download(e2e_cell.h, *host_out)
    # timed: repeated calls of K steps, each from the host fields to the host fields, enough calls
    # for ~200 steps in all (one call of K = 20 lasts ~10 ms, where host-side jitter shows)
    e2e_calls = max(1, -(-200 // max(args.steps, 1)))
    e2e_steps = 0
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_calls):
        lib.kks_upload(e2e_cell.h, *host_in)
        e2e_cell.run(args.steps)
        recs, rows = e2e_cell.drain()
        lib.kks_download(e2e_cell.h, *host_out)
        e2e_steps += e2e_cell.state().istep
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_cell.close()
    e2e_value = world * e2e_steps / e2e_s

    units = UNITS_ARMED if armed else UNITS_UNARMED
    peak, peak_kind = measured_peaks()
    alg_bytes = units * N * p
    achieved = alg_bytes / (ms_per_attempt / 1000.0) / 1e9
    traffic = None
    tpath = os.path.join(REPO, "profiles", f"attempt_traffic_1420_{args.precision}.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get("dram_bytes_per_attempt")

    # every rank takes part in the sharded ensemble leg (its barrier and max over ranks)
    sharded = None
    if world > 1 and not args.no_ensemble and args.precision != "fp64":
        sharded = sharded_ensemble_leg(args.precision, local_rank, 20, 3, rank, world, barrier, max_over_ranks)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_ms / max(steps_done, 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic",
        "config": bench_config(armed),
        "precision": args.precision,
        "attempts": int(attempts),
        "launch_shape": shape,
        "autotune": (None if tuned is None else {"ms_per_attempt": tuned["ms_per_attempt"],
                                                 "note": "fastest of the candidate shapes, timed on the cell "
                                                         "before the run"}),
        "cell_updates_per_s": value * N,
        "fp64_steps_per_s": fp64,
        "fp64_launch_shape": fp64_shape,
        "mixed_over_fp64": (value / world / fp64) if fp64 else None,
        "fp64_cufft_steps_per_s": fp64_cufft,
        "mixed_over_fp64_cufft": (value / world / fp64_cufft) if fp64_cufft else None,
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "kernel": (f"one attempt (captured CUDA graph of {kernels_per_attempt} kernels: shared-memory FFT passes "
                       "fused with the pointwise stages)") if fused else
                      "one attempt (captured CUDA graph: 8 own kernels + cuFFT R2C/C2R)",
            "algorithmic_bytes": alg_bytes,
            "peak_kind": peak_kind,
        },
        "clocks": clocks.summary(),
        "e2e": {
            "value": e2e_value,
            "unit": UNIT,
            "h2d_bytes_per_step": e2e_calls * 4 * N * 8 / max(e2e_steps, 1),
            "d2h_bytes_per_step": e2e_calls * (4 * N * 8 + len(rows) * 256 + len(recs) * 128) / max(e2e_steps, 1),
            "calls": e2e_calls,
            "steps_per_call": args.steps,
            "note": "kks_upload (4 fields) + kks_run(K) + kks_drain + kks_download (4 fields) per call of K steps",
        },
        "gpu_launches": int(kernels_per_attempt * attempts),
    }
    if not args.no_ensemble and args.precision != "fp64":
        if world == 1:
            line["ensemble"] = ensemble_leg(args.precision, local_rank, steps=20, warmup=3,
                                            cpu=not args.no_cpu_baseline)
        else:
            line["ensemble_sharded"] = sharded
    if long_run is not None:
        line["long_run"] = long_run
    if world == 1 and args.precision != "fp64" and not args.no_armed:
        line["armed_attempts"] = armed_leg(args.precision, local_rank, tables, peak)
    if not args.no_init and world == 1 and args.precision != "fp64":
        line["init"] = init_leg(args.precision, local_rank)
    if not args.no_adjoint and world == 1:
        line["adjoint"] = adjoint_leg(local_rank)
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(state, cfg)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
