"""Time integration of the extended KKS model on one B200: drop-in for
``pf_kks.solver`` (``pf_kks/solver.py:40-414``).

``run`` keeps the reference's signature, outputs and errors. Underneath, the
whole attempt loop runs on the GPU through ``libkks_b200.so`` (C ABI of
``include/kks.h``): the fields are uploaded once, every attempt (free energy,
elasticity, spectral Allen-Cahn / Cahn-Hilliard updates, phase compositions,
energy residual and the reject / accept / enlarge decision) runs on the
device, and the host only

* launches batches of steps up to the next map step (no synchronisation per
  attempt),
* formats the device's log records into ``log.txt`` / ``dtime.txt``
  (:mod:`pf_kks_gpu.runlog`) and its history rows into the history lists,
* downloads the fields at map steps and at the end.

``precision`` is taken from ``cfg.gpu`` (``[gpu]`` TOML section) unless given.
"""

import ctypes
import datetime
import os
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .io import map_filename, save_map
from .kinetics import quenched_vacancy_fraction
from .materials import TABLE_ORDER, MaterialTables
from .runlog import RunLog

HIST_NAMES = ("deta_mean", "eta_mean", "T", "dT", "dtime", "time", "time_s", "surf", "X_al_mean", "X_th_mean",
              "X_mean", "G_mean", "dX_al_mean", "dX_th_mean", "dsurf", "L")
RES_NAMES = ("total", "energy_derivative", "diffusion", "allen_cahn", "temperature")


@dataclass
class Schedule:
    """Steps at which outputs are produced (pf_kks/solver.py:40-53)."""

    n_steps: int
    map_steps: set
    surface_steps: set

    @classmethod
    def from_config(cls, cfg):
        map_steps = np.linspace(1, int(cfg.n_steps), cfg.n_map_saves, dtype=int)
        last = cfg.surface_sample_last_step or cfg.n_steps
        surface_steps = np.linspace(1, int(last), cfg.n_surface_samples, dtype=int)
        return cls(int(np.max(map_steps)), set(map_steps.tolist()), set(surface_steps.tolist()))


@dataclass
class SimulationResult:
    """Final fields and per-step histories (pf_kks/solver.py:56-69)."""

    X: np.ndarray
    X_al: np.ndarray
    X_th: np.ndarray
    eta: np.ndarray
    sig_el: np.ndarray
    eps_el: np.ndarray
    good_step: int | None
    ttime: float
    map_files: list = field(default_factory=list)
    history: dict = field(default_factory=dict)


class AdaptiveStepError(RuntimeError):
    """Raised when the adaptive time stepping cannot find an admissible step
    (pf_kks/solver.py:72-73)."""


@dataclass
class Residual:
    total: float
    energy_derivative: float
    diffusion_term: float
    allen_cahn_term: float
    temperature_term: float


def make_params(cfg, tables):
    """kks_params from a configuration and its tables, with the scaling that
    pf_kks/solver.py:101-116 applies at the start of a run."""
    p = L.KksParams()
    p.nx, p.ny = int(cfg.nx), int(cfg.ny)
    p.max_iterations = int(cfg.max_iterations)
    p.good_step_offset = int(cfg.good_step_offset)
    p.dx = float(cfg.dx)
    p.lambd = float(cfg.lambd)
    p.alpha = float(cfg.alpha)
    p.D0 = float((tables.D0 if cfg.D0 is None else cfg.D0) * cfg.c_D)
    p.QD = float(tables.QD if cfg.QD is None else cfg.QD)
    p.Meta0 = float(cfg.Meta0 * cfg.c_Meta)
    p.QMeta = float(cfg.QMeta)
    p.Lv2 = float(cfg.vacancy_sink_distance**2)
    p.diffusion_enhancement_cap = float(cfg.diffusion_enhancement_cap)
    p.Xv0 = float(quenched_vacancy_fraction(cfg.T_quench))
    p.dtime_s = float(cfg.dtime_s)
    p.dtime_max = float(cfg.dtime_max)
    p.dtime_min_divisor = float(cfg.dtime_min_divisor)
    p.residual_max = float(cfg.residual_max)
    p.residual_min = float(cfg.residual_min)
    p.step_factor = float(cfg.step_factor)
    p.x_equilibrium = float(cfg.x_equilibrium)
    p.surf_scale = float(cfg.dx**2 / (2 * cfg.lambd))
    st = np.asarray(cfg.schedule_time, dtype=np.float64)
    sT = np.asarray(cfg.schedule_temperature, dtype=np.float64)
    if st.ndim != 1 or st.shape != sT.shape or not 1 <= st.size <= L.KKS_MAX_SCHED:
        raise ValueError("schedule_time / schedule_temperature must be equal-length 1-D lists of 1..64 entries")
    p.n_sched = st.size
    p.sched_time[:st.size] = st.tolist()
    p.sched_temp[:st.size] = sT.tolist()
    tT = np.asarray(tables.T, dtype=np.float64)
    if not 1 <= tT.size <= L.KKS_MAX_TABLE:
        raise ValueError("material tables must have 1..32 temperatures")
    p.n_table = tT.size
    p.table_T[:tT.size] = tT.tolist()
    for k, name in enumerate(TABLE_ORDER):
        p.table[k][:tT.size] = np.asarray(getattr(tables, name), dtype=np.float64).tolist()
    return p


class Cell:
    """One simulation cell resident on one GPU (a kks_handle)."""

    def __init__(self, cfg, tables, precision="fp64", device=0, schedule=None, record_capacity=1 << 15):
        self.lib = L.load()
        self.nx, self.ny = int(cfg.nx), int(cfg.ny)
        self.N = self.nx * self.ny
        schedule = schedule or Schedule.from_config(cfg)
        self.n_steps = schedule.n_steps
        flags = np.zeros(max(self.n_steps, 1), dtype=np.uint8)
        for s in schedule.surface_steps:
            if 1 <= s <= self.n_steps:
                flags[s - 1] |= 1
        self._flags = flags
        prec = {"fp64": L.KKS_PRECISION_FP64, "mixed": L.KKS_PRECISION_MIXED,
                "mixed-cufft": L.KKS_PRECISION_MIXED_CUFFT}[precision]
        self.precision = precision
        self.params = make_params(cfg, tables)
        h = ctypes.c_void_p()
        L.check(self.lib.kks_create(ctypes.byref(self.params), prec, int(device), self.n_steps,
                                    flags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), int(record_capacity),
                                    ctypes.byref(h)), "kks_create")
        self.h = h

    def upload(self, eta, X, X_al, X_th):
        a = [L.as_field(v, self.N) for v in (eta, X, X_al, X_th)]
        L.check(self.lib.kks_upload(self.h, *(L.dptr(v) for v in a)), "kks_upload")

    def run(self, n_steps):
        st = ctypes.c_int32(0)
        L.check(self.lib.kks_run(self.h, int(n_steps), ctypes.byref(st)), "kks_run")
        return st.value

    def drain(self):
        s = self.state()
        nr, nw = int(s.n_records), int(s.n_rows)
        recs = (L.KksRecord * max(nr, 1))()
        rows = np.zeros((max(nw, 1), 32), dtype=np.float64)
        got_r, got_w = ctypes.c_int64(0), ctypes.c_int64(0)
        L.check(self.lib.kks_drain(self.h, recs, nr, ctypes.byref(got_r),
                                   rows.ctypes.data_as(ctypes.POINTER(L.KksStepRow)), nw, ctypes.byref(got_w)),
                "kks_drain")
        return list(recs[: got_r.value]), rows[: got_w.value]

    def state(self):
        s = L.KksRunState()
        L.check(self.lib.kks_get_state(self.h, ctypes.byref(s)), "kks_get_state")
        return s

    def download(self):
        out = [np.empty((self.nx, self.ny, 1), dtype=np.float64) for _ in range(4)]
        L.check(self.lib.kks_download(self.h, *(L.dptr(v) for v in out)), "kks_download")
        return tuple(out)  # eta, X, X_al, X_th

    def set_wait_polls(self, polls):
        """Poll count of the first bounded wait of the fused passes (a test
        hook for the timeout path; negative restores the default)."""
        L.check(self.lib.kks_set_wait_polls(self.h, int(polls)), "kks_set_wait_polls")

    def download_pair(self):
        """The minus entry of the energy residual's pair: (eta-, X-, mu-, G-),
        each (nx, ny, 1) float64 (kks_download_pair)."""
        out = [np.empty((self.nx, self.ny, 1), dtype=np.float64) for _ in range(4)]
        L.check(self.lib.kks_download_pair(self.h, *(L.dptr(v) for v in out)), "kks_download_pair")
        return tuple(out)

    def elastic_fields(self):
        """sig_el, eps_el with shape (3, 3, nx, ny, 1)."""
        s4 = np.empty((4, self.nx, self.ny), dtype=np.float64)
        e4 = np.empty((4, self.nx, self.ny), dtype=np.float64)
        L.check(self.lib.kks_elastic_fields(self.h, L.dptr(s4), L.dptr(e4)), "kks_elastic_fields")
        sig = np.zeros((3, 3, self.nx, self.ny, 1))
        eps = np.zeros((3, 3, self.nx, self.ny, 1))
        for t4, full in ((s4, sig), (e4, eps)):
            full[0, 0, ..., 0], full[1, 1, ..., 0], full[2, 2, ..., 0] = t4[0], t4[1], t4[2]
            full[0, 1, ..., 0] = full[1, 0, ..., 0] = t4[3]
        return sig, eps

    def checkpoint(self):
        size = ctypes.c_size_t(0)
        L.check(self.lib.kks_checkpoint(self.h, None, 0, ctypes.byref(size)), "kks_checkpoint")
        buf = (ctypes.c_char * size.value)()
        L.check(self.lib.kks_checkpoint(self.h, buf, size.value, ctypes.byref(size)), "kks_checkpoint")
        return bytes(buf)

    def restore(self, blob):
        buf = ctypes.create_string_buffer(blob, len(blob))
        L.check(self.lib.kks_restore(self.h, buf, len(blob)), "kks_restore")

    def timing(self):
        ms = ctypes.c_double(0)
        n = ctypes.c_int64(0)
        L.check(self.lib.kks_timing(self.h, ctypes.byref(ms), ctypes.byref(n)), "kks_timing")
        return ms.value, n.value

    def pipeline(self):
        """(fused, kernels): 1 if the attempt runs the shared-memory FFT passes,
        and the kernels of this library one attempt launches."""
        fused = ctypes.c_int32(0)
        kernels = ctypes.c_int32(0)
        L.check(self.lib.kks_pipeline(self.h, ctypes.byref(fused), ctypes.byref(kernels)), "kks_pipeline")
        return bool(fused.value), int(kernels.value)

    # -- launch shapes ------------------------------------------------------

    def launch_shape(self):
        """{"pipeline": 1 fused / 0 cuFFT, "cols": fused column tile,
        "field_blocks": grid of the grid-stride kernels}."""
        s = L.KksLaunchShape()
        L.check(self.lib.kks_get_launch_shape(self.h, ctypes.byref(s)), "kks_get_launch_shape")
        return {"pipeline": s.pipeline, "cols": s.cols, "field_blocks": s.field_blocks}

    def set_launch_shape(self, pipeline, cols, field_blocks):
        s = L.KksLaunchShape(int(pipeline), int(cols), int(field_blocks), 0)
        L.check(self.lib.kks_set_launch_shape(self.h, ctypes.byref(s)), "kks_set_launch_shape")

    def autotune(self, attempts=20, batchable=False):
        """Time every candidate launch shape on the current state (restored
        afterwards) and keep the fastest; returns (shape, ms per attempt).
        ``batchable``: only shapes with which the cell can join a batch."""
        s = L.KksLaunchShape()
        ms = ctypes.c_double(0)
        flags = L.KKS_TUNE_BATCHABLE if batchable else 0
        L.check(self.lib.kks_autotune(self.h, int(attempts), flags, ctypes.byref(s), ctypes.byref(ms)),
                "kks_autotune")
        return {"pipeline": s.pipeline, "cols": s.cols, "field_blocks": s.field_blocks}, ms.value

    # -- initial state written on the device (no nx*ny host arrays) ---------

    def voronoi_edges(self, seeds):
        """Periodic Voronoi labels of ``seeds`` ((n, 2), in cells) on the
        device; returns the number of edge pixels."""
        seeds = np.ascontiguousarray(seeds, dtype=np.float64).reshape(-1, 2)
        n = ctypes.c_int64(0)
        L.check(self.lib.kks_voronoi_edges(self.h, seeds.shape[0], L.dptr(seeds), ctypes.byref(n)),
                "kks_voronoi_edges")
        return int(n.value)

    def generate_fields(self, pick, jitter, radii, w, x_matrix, noise_low, noise_range, x_particle, rng_state,
                        pc_shift, pc_ratio, picks_are_points=False):
        """Diffuse particles, noisy matrix and phase compositions into the
        state; ``rng_state`` is numpy's PCG64 state dict before the noise."""
        pick = np.ascontiguousarray(pick, dtype=np.int64)
        jitter = np.ascontiguousarray(jitter, dtype=np.float64).reshape(-1, 2)
        radii = np.ascontiguousarray(radii, dtype=np.float64)
        a = L.KksGenArgs()
        a.n_particles = pick.size
        a.picks_are_points = int(bool(picks_are_points))
        a.pick = pick.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        a.jitter = L.dptr(jitter)
        a.radii = L.dptr(radii)
        a.w, a.x_matrix, a.noise_low, a.noise_range, a.x_particle = w, x_matrix, noise_low, noise_range, x_particle
        st = rng_state["state"]
        mask = (1 << 64) - 1
        a.rng_state[0], a.rng_state[1] = st["state"] & mask, st["state"] >> 64
        a.rng_inc[0], a.rng_inc[1] = st["inc"] & mask, st["inc"] >> 64
        a.pc_shift, a.pc_ratio = pc_shift, pc_ratio
        L.check(self.lib.kks_generate_fields(self.h, ctypes.byref(a)), "kks_generate_fields")

    @staticmethod
    def _circles(r, ox, oy, oz):
        arrs = [np.ascontiguousarray(v, dtype=np.float64).ravel() for v in (r, ox, oy, oz)]
        if len({a.size for a in arrs}) != 1:
            raise ValueError("r, ox, oy, oz must have the same length")
        return arrs

    def place_precipitates(self, dx, dy, x_matrix, x_precipitate, r, ox, oy, oz):
        """State = (eta, X, X_matrix, X_precipitate) of sharp circles
        (pf_kks/microstructure.py:7-52) written on the device."""
        arrs = self._circles(r, ox, oy, oz)
        L.check(self.lib.kks_place_precipitates(self.h, dx, dy, x_matrix, x_precipitate, arrs[0].size,
                                                *(L.dptr(a) for a in arrs)), "kks_place_precipitates")

    def add_nuclei(self, dx, dy, r, ox, oy, oz):
        """Nuclei into the current state, in place (pf_kks/microstructure.py:55-74)."""
        arrs = self._circles(r, ox, oy, oz)
        L.check(self.lib.kks_add_nuclei(self.h, dx, dy, arrs[0].size, *(L.dptr(a) for a in arrs)),
                "kks_add_nuclei")

    def count_below(self, eta_below):
        """Number of points of the current state with eta < eta_below."""
        n = ctypes.c_int64(0)
        L.check(self.lib.kks_count_below(self.h, float(eta_below), ctypes.byref(n)), "kks_count_below")
        return int(n.value)

    def insert_nuclei(self, ranks, eta_below):
        """eta = 1 at the ranks-th points (C order) with eta < eta_below."""
        ranks = np.ascontiguousarray(np.atleast_1d(ranks), dtype=np.int64)
        L.check(self.lib.kks_insert_nuclei(self.h, float(eta_below), ranks.size,
                                           ranks.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
                "kks_insert_nuclei")

    def close(self):
        if getattr(self, "h", None):
            self.lib.kks_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def raise_for_status(cell, status):
    """The error a stopped cell reports: AdaptiveStepError with the reference's
    messages for its two stops (pf_kks/solver.py:292-295, 312-313), KksError
    when a bounded device wait ran out."""
    if status == L.KKS_STATUS_OK:
        return
    s = cell.state()
    if status == L.KKS_STATUS_TIMEOUT:
        raise L.KksError(f"step {s.istep}: a bounded device wait ran out (bulk copy not completed)")
    if status == L.KKS_STATUS_MAX_ITER:
        raise AdaptiveStepError(f"step {s.error_istep}: no admissible time step after "
                                f"{s.error_iteration} attempts (dtime_s={s.error_dtime_s:.2e})")
    raise AdaptiveStepError(f"step {s.error_istep}: non-finite energy residual")


def _residual(r):
    return Residual(r.res_total, r.res_energy_derivative, r.res_diffusion, r.res_allen_cahn, r.res_temperature)


class _HistoryBuilder:
    """Turns device records and rows into the reference's logs, prints and
    history lists (including its Python scalar types: ``time[0]`` is the int 0
    and ``time_s`` stays integral while every step size is an int)."""

    def __init__(self, cfg, log, verbose, nstep):
        self.cfg = cfg
        self.log = log
        self.verbose = verbose
        self.hist = {name: [] for name in HIST_NAMES}
        self.energy = np.zeros(nstep)
        self.dtime_s = np.zeros(nstep)
        self.res = {name: np.zeros(nstep) for name in RES_NAMES}
        self.dtime_s_min = cfg.dtime_s / cfg.dtime_min_divisor
        self.prev_dt = cfg.dtime_s
        self.prev_dt_int = isinstance(cfg.dtime_s, int)
        self.ts_int = True
        self.float_steps = set()

    def records(self, recs):
        cfg = self.cfg
        for r in recs:
            if r.kind == L.KKS_REC_STATE:
                self.log.state(r.istep, r.T, r.D, r.L, r.Meta, r.Vm, r.dtime_s)
                continue
            res = _residual(r)
            self.float_steps.add(r.istep)
            if self.verbose and r.istep % 1000 == 0:
                print("step, |RES-KKS|  , energy_term , gradient_term, eta_term, temp_term : ", r.istep,
                      "{0:.2e}".format(np.abs(res.total)), "{0:.2e}".format(res.energy_derivative),
                      "{0:.2e}".format(res.diffusion_term), "{0:.2e}".format(res.allen_cahn_term),
                      "{0:.2e}".format(res.temperature_term))
            if self.verbose and r.istep == r.good_step + 2 and r.iteration == 1:
                print("resmax= ", "{0:.2e}".format(cfg.residual_max), " resmin= ", "{0:.2e}".format(cfg.residual_min),
                      "\n")
                print("good step: ", r.good_step, "\n")
            if r.kind == L.KKS_REC_REJECTED:
                self.log.rejected(r.istep, r.iteration, r.dtime_s, res, r.energy_s)
            elif r.kind == L.KKS_REC_ACCEPTED:
                self.log.accepted(r.istep, res, r.energy_s)
            elif r.kind == L.KKS_REC_ENLARGED:
                self.log.enlarged(r.istep, res, r.energy_s)

    def _dt_is_int(self, istep):
        if istep == 0:
            v, is_int = self.cfg.dtime_s, isinstance(self.cfg.dtime_s, int)
        else:
            v, is_int = self.prev_dt, self.prev_dt_int
        if v > self.cfg.dtime_max:
            is_int = isinstance(self.cfg.dtime_max, int)
        elif v < self.dtime_s_min:
            is_int = False
        if istep in self.float_steps:  # a rejection or an enlargement divided / multiplied it
            is_int = False
        return is_int

    def rows(self, rows):
        H = L.H
        hist = self.hist
        for v in rows:
            istep = int(v[H["istep"]])
            f = np.float64
            is_int = self._dt_is_int(istep)
            self.prev_dt, self.prev_dt_int = float(v[H["dtime_s"]]), is_int
            self.ts_int = self.ts_int and is_int
            hist["X_al_mean"].append(f(v[H["X_al_mean"]]))
            hist["X_th_mean"].append(f(v[H["X_th_mean"]]))
            hist["X_mean"].append(f(v[H["X_mean"]]))
            hist["dX_al_mean"].append(f(v[H["dX_al_mean"]]))
            hist["dX_th_mean"].append(f(v[H["dX_th_mean"]]))
            hist["deta_mean"].append(f(v[H["deta_mean"]]))
            hist["dT"].append(f(v[H["dT"]]))
            hist["eta_mean"].append(f(v[H["eta_mean"]]))
            hist["G_mean"].append(f(v[H["G_mean"]]))
            hist["surf"].append(f(v[H["surf"]]))
            hist["dsurf"].append(f(v[H["dsurf"]]))
            hist["T"].append(f(v[H["T"]]))
            hist["dtime"].append(f(v[H["dtime"]]))
            hist["time"].append(0 if istep == 0 else f(v[H["time"]]))
            ts = v[H["time_s"]]
            hist["time_s"].append(int(ts) if self.ts_int else float(ts))
            hist["L"].append(f(v[H["L"]]))
            self.energy[istep] = v[H["energy_s"]]
            self.dtime_s[istep] = v[H["dtime_s"]]
            for k, name in enumerate(RES_NAMES):
                self.res[name][istep] = v[H["residual_total"] + k]


def run(cfg, eta, X, X_al, X_th, out_dir=".", base_dir=".", write_logs=True, verbose=True, precision=None,
        device=None):
    """Run the simulation on the GPU (signature of pf_kks/solver.py:76-98).

    Parameters and outputs are those of the reference. ``precision`` ("fp64" or
    "mixed") and ``device`` override ``cfg.gpu``.
    """
    t_wall = time.time()
    opts = cfg.gpu_options
    precision = precision or opts.precision
    device = opts.device if device is None else device
    log = RunLog(out_dir, enabled=write_logs)
    maps_dir = os.path.join(out_dir, "saved_maps")
    os.makedirs(maps_dir, exist_ok=True)
    if cfg.nz != 1:
        raise ValueError("the GPU step is 2-D (nz = 1), like the reference's energy and residual")
    tables = MaterialTables.from_npz(cfg.resolve_path(cfg.material_tables, base_dir), cfg.c_gamma, cfg.c_eps0)
    schedule = Schedule.from_config(cfg)
    nstep = schedule.n_steps
    cell = Cell(cfg, tables, precision=precision, device=device, schedule=schedule,
                record_capacity=opts.records_capacity)
    hb = _HistoryBuilder(cfg, log, verbose, nstep)
    map_files = []
    try:
        cell.upload(eta, X, X_al, X_th)
        if opts.autotune and nstep >= 2:
            from . import autotune

            autotune.tune(cell, device=device)
        stops = sorted(s for s in schedule.map_steps if 1 <= s <= nstep)
        if not stops or stops[-1] != nstep:
            stops.append(nstep)
        done = 0
        for stop in stops:
            status = cell.run(stop - done)
            recs, rows = cell.drain()
            hb.records(recs)
            hb.rows(rows)
            log.flush()
            raise_for_status(cell, status)
            done = stop
            if stop in schedule.map_steps:
                e, x, xa, xt = cell.download()
                s = cell.state()
                name = map_filename(s.ttime, cfg.T_start, np.asarray(hb.hist["T"]).max())
                path = os.path.join(maps_dir, name)
                save_map(path, s.ttime, hb.hist, x, xa, xt, e)
                map_files.append(path + ".npz")
        eta_f, X_f, X_al_f, X_th_f = cell.download()
        sig_el, eps_el = cell.elastic_fields() if nstep > 0 else (None, None)
        s = cell.state()
        good_step = int(s.good_step) if s.flag else None
        ttime = float(s.ttime)
    finally:
        cell.close()

    if verbose:
        print("Temperature reached : %s K ---" % (np.asarray(hb.hist["T"]).max()))
        print("simulation time : " + str(datetime.timedelta(seconds=time.time() - t_wall)))
    hist = hb.hist
    hist["energy_s"] = hb.energy
    hist["dtime_s"] = hb.dtime_s
    for name, values in hb.res.items():
        hist["residual_" + name] = values
    return SimulationResult(X_f, X_al_f, X_th_f, eta_f, sig_el, eps_el, good_step, ttime, map_files, hist)
