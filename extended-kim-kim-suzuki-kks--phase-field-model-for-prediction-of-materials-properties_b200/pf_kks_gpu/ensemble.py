"""Ensembles of independent cells: sharding across GPUs and concurrent cells
on one GPU.

Cells of an ensemble (different sizes, seeds, heating rates) share nothing, so
the multi-GPU layout is a partition of the cells over ranks, one process per
GPU, with no collective inside the step; per-cell results are gathered on the
host at the end. On one GPU the cells of a shard run as concurrent attempt
graphs on their own streams (each cell keeps its own adaptive dt, rejection and
device loop state), so small grids that cannot fill 148 SMs alone overlap.
"""

import math
import time

import numpy as np


def cell_cost(nx, ny, steps=1):
    """Relative cost of a cell: N log N of its transforms times its steps."""
    n = nx * ny
    return steps * n * max(math.log2(n), 1.0)


def partition(costs, world):
    """Longest-processing-time assignment of cells to ``world`` ranks.

    Returns a list of ``world`` lists of cell indices; deterministic (ties go
    to the lower rank, cells are taken by decreasing cost then index).
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += costs[i]
    for s in shards:
        s.sort()
    return shards


def gather_results(local, group=None):
    """All-gather a picklable per-rank result dict {cell index: result} over
    ``torch.distributed`` (NCCL or gloo); returns the merged dict on every
    rank. Without an initialised process group, returns ``local``."""
    try:
        import torch.distributed as dist
    except Exception:  # torch absent: single process
        return dict(local)
    if not dist.is_available() or not dist.is_initialized():
        return dict(local)
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, local, group=group)
    merged = {}
    for part in out:
        merged.update(part)
    return merged


def run_shard(cells, n_steps, device=0):
    """Advance every (cfg, tables, state) cell of this shard by ``n_steps``
    steps on one GPU, interleaving their batches so that cells overlap.

    Returns {index: dict(status, steps, attempts, device_ms, fields)}.
    """
    from .solver import Cell

    handles = {}
    for idx, (cfg, tables, state) in cells.items():
        c = Cell(cfg, tables, precision=cfg.gpu_options.precision, device=device)
        c.upload(*state)
        handles[idx] = c
    t0 = time.perf_counter()
    out = {}
    for idx, c in handles.items():
        st = c.run(n_steps)
        c.drain()
        s = c.state()
        ms, att = c.timing()
        out[idx] = {"status": st, "steps": int(s.istep), "attempts": int(s.attempts), "device_ms": ms,
                    "eta": None, "X": None}
    wall = time.perf_counter() - t0
    for idx, c in handles.items():
        e, x, _, _ = c.download()
        out[idx]["eta_mean"] = float(np.mean(e))
        out[idx]["X_mean"] = float(np.mean(x))
        c.close()
    return out, wall
