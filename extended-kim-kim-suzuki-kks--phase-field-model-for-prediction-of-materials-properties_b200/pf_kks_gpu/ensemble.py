"""Ensembles of independent cells: sharding across GPUs and concurrent cells
on one GPU.

Cells of an ensemble (different sizes, seeds, heating rates) share nothing, so
the multi-GPU layout is a partition of the cells over ranks, one process per
GPU, with no collective inside the step; per-cell results are gathered on the
host at the end. On one GPU the cells of a shard advance as one batch
(``kks_batch_run``): every kernel of an attempt is launched once for all cells
over their device descriptors, one CUDA graph per batch attempt, while each
cell keeps its own adaptive dt, rejections, step target and buffer parity on
the device. Cells that cannot share a batch (the cuFFT or FP64 pipelines, or
different large prime factors) run as concurrent attempt graphs on their own
streams (``kks_run_many``).
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


def _rank_world():
    try:
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(), dist.get_world_size()
    except Exception:
        pass
    return 0, 1


def run_sharded(members, n_steps, precision="mixed", device=None, tune=False, fields=False, rank=None, world=None,
                make_ensemble=None):
    """Run an ensemble over the ranks of a job, one process per GPU.

    ``members``: the whole ensemble, a list of (cfg, state) pairs on every
    rank (``state`` may be a callable returning the four fields, so that a
    rank builds only its own cells). The cells are partitioned by cost
    (:func:`partition`, cost = N log N x steps); this rank advances its shard
    as one :class:`Ensemble` on ``device`` (default: $LOCAL_RANK) by
    ``n_steps`` (an int or one count per member); the per-cell results
    (:meth:`Ensemble.results`) are then gathered on every rank with one
    all-gather. There is no collective inside the steps. ``rank`` / ``world``
    default to the initialised process group (else 0 / 1); ``make_ensemble``
    replaces the Ensemble class (tests). Returns (results by member index,
    this rank's shard, its status list)."""
    import os

    if rank is None or world is None:
        rank, world = _rank_world()
    if device is None:
        device = int(os.environ.get("LOCAL_RANK", 0))
    counts = [int(n_steps)] * len(members) if np.isscalar(n_steps) else [int(k) for k in n_steps]
    costs = [cell_cost(cfg.nx, cfg.ny, k) for (cfg, _), k in zip(members, counts)]
    shard = partition(costs, world)[rank]
    local = {}
    status = []
    if shard:
        cells = [(members[i][0], members[i][1]() if callable(members[i][1]) else members[i][1]) for i in shard]
        ens = (make_ensemble or Ensemble)(cells, precision=precision, device=device, tune=tune)
        try:
            status = ens.run([counts[i] for i in shard])
            for i, r in zip(shard, ens.results(fields=fields)):
                r["rank"] = rank
                local[i] = r
        finally:
            ens.close()
    return gather_results(local), shard, status


class Ensemble:
    """Cells of one shard resident on one GPU, advanced together.

    ``batched``: None (default) batches the cells when they allow it and
    otherwise runs them on their own streams; True requires the batch (raises
    if the cells cannot share one); False always uses the per-cell streams.
    ``mode`` tells which one is in use ("batch" or "streams").
    ``cols``: a fused column tile for every cell (instead of the default).
    ``groups``: the batch's cells are split into that many groups of about
    equal cost, each a graph on its own stream (their passes overlap).
    ``tune``: choose the launch shapes first. For a batch, the column tile of
    the fused column passes and then the number of groups are timed on the
    batch itself (the cells' states are saved before and restored after every
    candidate), because a tile that is best for a small cell alone (many small
    blocks to fill the GPU) wastes SM slots when all cells share the grid.
    Cells on their own streams get the autotuner's shape of the first cell of
    each grid size. ``shapes``, ``groups`` and ``batch_tile_ms`` /
    ``batch_grid_ms`` / ``batch_groups_ms`` hold the choices and their device
    times per attempt.
    With ``tune`` and a batch, the batch and the per-cell streams are then
    timed on the same attempts (host wall clock, one synchronisation per
    call) and ``run`` uses the faster (``mode``; ``mode_ms`` holds the times).
    """

    def __init__(self, members, precision="mixed", device=0, batched=None, tune=False, tune_attempts=10,
                 groups=1, cols=None):
        import ctypes

        from . import _lib as L
        from .materials import MaterialTables
        from .solver import Cell

        self.cells = []
        for cfg, state in members:
            tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
            c = Cell(cfg, tables, precision=precision, device=device)
            c.upload(*state)
            self.cells.append(c)
        self.shapes = {}
        if cols is not None:
            for c in self.cells:
                c.set_launch_shape(1, cols, c.launch_shape()["field_blocks"])
        self._ptrs = (ctypes.c_void_p * len(self.cells))(*[c.h.value for c in self.cells])
        self.batch_tile_ms = {}
        self.batch_grid_ms = {}
        self.batch_groups_ms = {}
        self.groups = int(groups)
        tuned_batch = tune and batched is not False and self.cells and self._tune_batch(tune_attempts)
        if tune and not tuned_batch:
            from . import autotune

            for c in self.cells:
                k = (c.nx, c.ny)
                if k not in self.shapes:
                    self.shapes[k] = autotune.tune(c, attempts=tune_attempts, device=device, cache=False)["shape"]
                else:
                    c.set_launch_shape(**self.shapes[k])
        self.points = [c.N for c in self.cells]
        self.batch = None
        self.mode = "streams"
        self.mode_ms = {}
        if batched is not False and self.cells:
            b = ctypes.c_void_p()
            rc = L.load().kks_batch_create(self._ptrs, len(self.cells), self.groups, ctypes.byref(b))
            if rc == L.KKS_OK:
                self.batch = b
                self.mode = "batch"
            elif batched:
                L.check(rc, "kks_batch_create")
        if tuned_batch and batched is None:
            self._choose_mode(tune_attempts)
        # history rows of the run proper (tuning attempts are rolled back)
        self.rows = [[] for _ in self.cells]

    def _choose_mode(self, attempts):
        """Time the batch and the per-cell streams on the same attempts of the
        current state (restored afterwards) and keep the faster."""
        import time

        left = min(c.n_steps - c.state().istep for c in self.cells)
        k = min(int(attempts), left - 1)
        if k < 1:
            return
        blobs = [c.checkpoint() for c in self.cells]
        for mode, fn in (("batch", lambda m: self._call("kks_batch_run", (self.batch,), m)),
                         ("streams", self.run_streams)):
            fn(1)
            t0 = time.perf_counter()
            st = fn(k)
            dt = time.perf_counter() - t0
            for c, blob in zip(self.cells, blobs):
                c.restore(blob)
            if all(v == 0 for v in st):
                self.mode_ms[mode] = 1000.0 * dt / k
        if len(self.mode_ms) == 2:
            self.mode = min(self.mode_ms, key=self.mode_ms.get)

    def _time_batch(self, groups, k, blobs):
        """Device ms per batch attempt of the cells' current shapes with the
        given groups (None if the cells cannot form that batch); the cells'
        states are restored from ``blobs`` afterwards."""
        import ctypes

        from . import _lib as L

        lib = L.load()
        n = len(self.cells)
        b = ctypes.c_void_p()
        if lib.kks_batch_create(self._ptrs, n, int(groups), ctypes.byref(b)) != L.KKS_OK:
            return None
        per = None
        try:
            st = (ctypes.c_int32 * n)()
            L.check(lib.kks_batch_run(b, (ctypes.c_int32 * n)(*([1] * n)), st), "kks_batch_run")
            ms0, a0 = ctypes.c_double(), ctypes.c_int64()
            L.check(lib.kks_batch_timing(b, ctypes.byref(ms0), ctypes.byref(a0)), "kks_batch_timing")
            L.check(lib.kks_batch_run(b, (ctypes.c_int32 * n)(*([k] * n)), st), "kks_batch_run")
            ms1, a1 = ctypes.c_double(), ctypes.c_int64()
            L.check(lib.kks_batch_timing(b, ctypes.byref(ms1), ctypes.byref(a1)), "kks_batch_timing")
            if a1.value > a0.value and all(v == L.KKS_STATUS_OK for v in st):
                per = (ms1.value - ms0.value) / (a1.value - a0.value)
        finally:
            L.check(lib.kks_batch_destroy(b), "kks_batch_destroy")
            for c, blob in zip(self.cells, blobs):
                c.restore(blob)
        return per

    def _tune_batch(self, attempts):
        """Time the batch with every column tile 1..4 (the same for all cells,
        field grids unchanged), then the field-kernel grids divided by 1, 4
        and 16, then 1, 2, 3 and 4 groups; keep the fastest of each. False if
        the cells cannot form a batch."""
        from . import _lib as L

        left = min(c.n_steps - c.state().istep for c in self.cells)
        k = min(int(attempts), left - 1)
        if k < 1:
            return False
        blobs = [c.checkpoint() for c in self.cells]
        grids = [c.launch_shape()["field_blocks"] for c in self.cells]
        for cols in (1, 2, 3, 4):
            try:
                for c, g in zip(self.cells, grids):
                    c.set_launch_shape(1, cols, g)
            except L.KksError:
                continue
            per = self._time_batch(1, k, blobs)
            if per is not None:
                self.batch_tile_ms[cols] = per
        if not self.batch_tile_ms:
            return False
        cols = min(self.batch_tile_ms, key=self.batch_tile_ms.get)
        # the grid-stride kernels (gradient energy, interface count, restore):
        # coarser grids than a cell alone wants, since 48 cells share the GPU
        self.batch_grid_ms = {1: self.batch_tile_ms[cols]}
        for d in (4, 16):
            for c, g in zip(self.cells, grids):
                c.set_launch_shape(1, cols, max(1, g // d))
            per = self._time_batch(1, k, blobs)
            if per is not None:
                self.batch_grid_ms[d] = per
        d = min(self.batch_grid_ms, key=self.batch_grid_ms.get)
        for c, g in zip(self.cells, grids):
            c.set_launch_shape(1, cols, max(1, g // d))
            self.shapes[(c.nx, c.ny)] = c.launch_shape()
        self.batch_groups_ms[1] = self.batch_grid_ms[d]
        for groups in (2, 3, 4):
            if groups <= len(self.cells):
                per = self._time_batch(groups, k, blobs)
                if per is not None:
                    self.batch_groups_ms[groups] = per
        self.groups = min(self.batch_groups_ms, key=self.batch_groups_ms.get)
        return True

    def run(self, n_steps):
        """Advance every cell by ``n_steps`` steps (an int, or one count per
        cell); returns the status per cell."""
        if self.mode == "batch":
            return self.run_batch(n_steps)
        return self.run_streams(n_steps)

    def run_batch(self, n_steps):
        """The same steps as one batch (``kks_batch_run``)."""
        if self.batch is None:
            raise RuntimeError("these cells do not form a batch")
        return self._call("kks_batch_run", (self.batch,), n_steps)

    def run_streams(self, n_steps):
        """The same steps with every cell on its own stream (``kks_run_many``)."""
        return self._call("kks_run_many", (self._ptrs, len(self.cells)), n_steps)

    def _call(self, fn, head, n_steps):
        import ctypes

        from . import _lib as L

        n = len(self.cells)
        counts = [int(n_steps)] * n if np.isscalar(n_steps) else [int(k) for k in n_steps]
        if len(counts) != n:
            raise ValueError(f"{len(counts)} step counts for {n} cells")
        steps = (ctypes.c_int32 * n)(*counts)
        status = (ctypes.c_int32 * n)()
        L.check(getattr(L.load(), fn)(*head, steps, status), fn)
        self._collect()
        return list(status)

    def _collect(self):
        """Drain every cell's device records, keeping its history rows."""
        if not hasattr(self, "rows"):
            self.rows = [[] for _ in self.cells]
        for k, c in enumerate(self.cells):
            _, rows = c.drain()
            if len(rows):
                self.rows[k].append(rows)

    def results(self, fields=False):
        """Per-cell results, in member order: the loop state (status, step,
        attempts, good_step or None, ttime), the history rows of all steps run
        so far ((steps, 32) float64, columns KKS_H_* of include/kks.h) and, with
        ``fields``, the final (eta, X, X_al, X_th)."""
        out = []
        for k, c in enumerate(self.cells):
            s = c.state()
            rows = getattr(self, "rows", [[]] * len(self.cells))[k]
            r = {"status": int(s.status), "istep": int(s.istep), "attempts": int(s.attempts),
                 "good_step": int(s.good_step) if s.flag else None, "ttime": float(s.ttime),
                 "rows": np.concatenate(rows) if rows else np.zeros((0, 32))}
            if fields:
                r["fields"] = c.download()
            out.append(r)
        return out

    def batch_timing(self):
        """(device ms, batch attempts) of all batched runs so far."""
        import ctypes

        from . import _lib as L

        if self.batch is None:
            return 0.0, 0
        ms, att = ctypes.c_double(), ctypes.c_int64()
        L.check(L.load().kks_batch_timing(self.batch, ctypes.byref(ms), ctypes.byref(att)), "kks_batch_timing")
        return ms.value, att.value

    def run_sequential(self, n_steps):
        """The same steps, one cell after the other (the comparison baseline)."""
        out = []
        for c in self.cells:
            out.append(c.run(n_steps))
        self._collect()
        return out

    def close(self):
        if self.batch is not None:
            from . import _lib as L

            L.check(L.load().kks_batch_destroy(self.batch), "kks_batch_destroy")
            self.batch = None
        for c in self.cells:
            c.close()
        self.cells = []
