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


class Ensemble:
    """Cells of one shard resident on one GPU, advanced together by
    ``kks_run_many`` (each cell on its own stream with its own graphs, one host
    synchronisation per batch for all of them)."""

    def __init__(self, members, precision="mixed", device=0):
        import ctypes

        from .materials import MaterialTables
        from .solver import Cell

        self.cells = []
        for cfg, state in members:
            tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
            c = Cell(cfg, tables, precision=precision, device=device)
            c.upload(*state)
            self.cells.append(c)
        self._ptrs = (ctypes.c_void_p * len(self.cells))(*[c.h.value for c in self.cells])
        self.points = [c.N for c in self.cells]

    def run(self, n_steps):
        """Advance every cell by ``n_steps`` steps; returns the status per cell."""
        import ctypes

        from . import _lib as L

        n = len(self.cells)
        steps = (ctypes.c_int32 * n)(*([int(n_steps)] * n))
        status = (ctypes.c_int32 * n)()
        L.check(L.load().kks_run_many(self._ptrs, n, steps, status), "kks_run_many")
        for c in self.cells:
            c.drain()
        return list(status)

    def run_sequential(self, n_steps):
        """The same steps, one cell after the other (the comparison baseline)."""
        out = []
        for c in self.cells:
            out.append(c.run(n_steps))
            c.drain()
        return out

    def close(self):
        for c in self.cells:
            c.close()
        self.cells = []
