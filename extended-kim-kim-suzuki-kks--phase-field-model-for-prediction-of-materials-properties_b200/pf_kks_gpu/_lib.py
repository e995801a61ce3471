"""ctypes binding of ``libkks_b200.so`` (declarations in ``include/kks.h``).

The library is the only compute path: if it is missing or no CUDA device can
be used, the calls below raise; nothing falls back to the CPU.
"""

import ctypes
import os

import numpy as np

LIB_NAME = "libkks_b200.so"
# $KKS_LIBRARY selects another build of the library (e.g. the bounds-check
# build libkks_b200_check.so of pf_kks_gpu.build --bounds-check)
LIB_PATH = os.environ.get("KKS_LIBRARY") or os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)
CHECK_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libkks_b200_check.so")

KKS_OK = 0
KKS_STATUS_OK = 0
KKS_STATUS_MAX_ITER = 1
KKS_STATUS_NONFINITE = 2
KKS_STATUS_TIMEOUT = 3
KKS_COEF_COUNT = 15
COEF_NAMES = ("dt", "L_s", "kappa2_s", "D_s", "w_s", "A_alp_s", "B_alp_s", "C_alp_s", "A_thet_s", "B_thet_s",
              "C_thet_s", "epsX", "C44", "pc_shift", "pc_ratio")
KKS_PRECISION_FP64 = 0
KKS_PRECISION_MIXED = 1
KKS_PRECISION_MIXED_CUFFT = 2
KKS_TUNE_BATCHABLE = 1
KKS_MAX_SCHED = 64
KKS_MAX_TABLE = 32
KKS_NTAB = 13

KKS_REC_STATE = 1
KKS_REC_REJECTED = 2
KKS_REC_ACCEPTED = 3
KKS_REC_ENLARGED = 4

# kks_step_row column indices (KKS_H_* in kks.h)
H = {
    name: i
    for i, name in enumerate(
        (
            "X_al_mean", "X_th_mean", "X_mean", "dX_al_mean", "dX_th_mean", "deta_mean", "dT", "eta_mean",
            "G_mean", "surf", "dsurf", "T", "dtime", "time", "time_s", "L", "energy_s", "dtime_s",
            "residual_total", "residual_energy_derivative", "residual_diffusion", "residual_allen_cahn",
            "residual_temperature", "ttime", "istep", "surf_valid", "D", "Xv",
        )
    )
}

# Exported symbols, one per declaration of include/kks.h.
EXPORTS = (
    "kks_create", "kks_upload", "kks_run", "kks_drain", "kks_get_state", "kks_download", "kks_elastic_fields",
    "kks_checkpoint", "kks_restore", "kks_timing", "kks_destroy", "kks_last_error", "kks_version",
    "kks_state_sums_noalloc", "kks_run_many", "kks_pipeline",
    "kks_adj_create", "kks_adj_forward", "kks_adj_backward", "kks_adj_destroy", "kks_adj_set_precision",
    "kks_adj_backward_device", "kks_adj_set_stream",
    "kks_voronoi_edges", "kks_generate_fields", "kks_place_precipitates", "kks_add_nuclei", "kks_count_below",
    "kks_insert_nuclei", "kks_batch_create", "kks_batch_run", "kks_batch_timing", "kks_batch_destroy",
    "kks_get_launch_shape", "kks_set_launch_shape", "kks_autotune", "kks_download_pair",
    "kks_set_wait_polls", "kks_bounds_report",
)


class KksLaunchShape(ctypes.Structure):
    _fields_ = [("pipeline", ctypes.c_int32), ("cols", ctypes.c_int32), ("field_blocks", ctypes.c_int32),
                ("pad", ctypes.c_int32)]


class KksParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("max_iterations", ctypes.c_int32), ("good_step_offset", ctypes.c_int32),
        ("dx", ctypes.c_double), ("lambd", ctypes.c_double), ("alpha", ctypes.c_double),
        ("D0", ctypes.c_double), ("QD", ctypes.c_double), ("Meta0", ctypes.c_double), ("QMeta", ctypes.c_double),
        ("Lv2", ctypes.c_double), ("diffusion_enhancement_cap", ctypes.c_double), ("Xv0", ctypes.c_double),
        ("dtime_s", ctypes.c_double), ("dtime_max", ctypes.c_double), ("dtime_min_divisor", ctypes.c_double),
        ("residual_max", ctypes.c_double), ("residual_min", ctypes.c_double), ("step_factor", ctypes.c_double),
        ("x_equilibrium", ctypes.c_double), ("surf_scale", ctypes.c_double),
        ("n_sched", ctypes.c_int32), ("n_table", ctypes.c_int32),
        ("sched_time", ctypes.c_double * KKS_MAX_SCHED), ("sched_temp", ctypes.c_double * KKS_MAX_SCHED),
        ("table_T", ctypes.c_double * KKS_MAX_TABLE),
        ("table", (ctypes.c_double * KKS_MAX_TABLE) * KKS_NTAB),
    ]


class KksRecord(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("istep", ctypes.c_int32), ("iteration", ctypes.c_int32),
        ("good_step", ctypes.c_int32),
        ("T", ctypes.c_double), ("D", ctypes.c_double), ("L", ctypes.c_double), ("Meta", ctypes.c_double),
        ("Vm", ctypes.c_double), ("dtime_s", ctypes.c_double),
        ("res_total", ctypes.c_double), ("res_energy_derivative", ctypes.c_double),
        ("res_diffusion", ctypes.c_double), ("res_allen_cahn", ctypes.c_double),
        ("res_temperature", ctypes.c_double), ("energy_s", ctypes.c_double),
    ]


class KksStepRow(ctypes.Structure):
    _fields_ = [("v", ctypes.c_double * 32)]


class KksRunState(ctypes.Structure):
    _fields_ = [
        ("istep", ctypes.c_int32), ("iteration", ctypes.c_int32), ("flag", ctypes.c_int32),
        ("good_step", ctypes.c_int32), ("status", ctypes.c_int32), ("parity", ctypes.c_int32),
        ("attempts", ctypes.c_int64), ("n_records", ctypes.c_int64), ("n_rows", ctypes.c_int64),
        ("t", ctypes.c_double), ("t_s", ctypes.c_double), ("t_b", ctypes.c_double), ("ttime", ctypes.c_double),
        ("Xv", ctypes.c_double), ("dtime_s", ctypes.c_double), ("D_0", ctypes.c_double),
        ("Meta_0", ctypes.c_double), ("surf", ctypes.c_double), ("surf_b", ctypes.c_double),
        ("T_b", ctypes.c_double),
        ("error_istep", ctypes.c_int32), ("error_iteration", ctypes.c_int32), ("error_dtime_s", ctypes.c_double),
    ]


class KksGenArgs(ctypes.Structure):
    _fields_ = [
        ("n_particles", ctypes.c_int32), ("picks_are_points", ctypes.c_int32),
        ("pick", ctypes.POINTER(ctypes.c_int64)), ("jitter", ctypes.POINTER(ctypes.c_double)),
        ("radii", ctypes.POINTER(ctypes.c_double)),
        ("w", ctypes.c_double), ("x_matrix", ctypes.c_double), ("noise_low", ctypes.c_double),
        ("noise_range", ctypes.c_double), ("x_particle", ctypes.c_double),
        ("rng_state", ctypes.c_uint64 * 2), ("rng_inc", ctypes.c_uint64 * 2),
        ("pc_shift", ctypes.c_double), ("pc_ratio", ctypes.c_double),
    ]


_lib = None


def load(path=LIB_PATH):
    """Load the shared library and declare its signatures (once)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m pf_kks_gpu.build` (nvcc, sm_100a). "
            "There is no CPU fallback."
        )
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    dp = P(ctypes.c_double)
    lib.kks_create.argtypes = [P(KksParams), ctypes.c_int, ctypes.c_int, ctypes.c_int32, P(ctypes.c_uint8),
                               ctypes.c_int64, P(vp)]
    lib.kks_upload.argtypes = [vp, dp, dp, dp, dp]
    lib.kks_run.argtypes = [vp, ctypes.c_int32, P(ctypes.c_int32)]
    lib.kks_drain.argtypes = [vp, P(KksRecord), ctypes.c_int64, P(ctypes.c_int64), P(KksStepRow), ctypes.c_int64,
                              P(ctypes.c_int64)]
    lib.kks_get_state.argtypes = [vp, P(KksRunState)]
    lib.kks_download.argtypes = [vp, dp, dp, dp, dp]
    lib.kks_download_pair.argtypes = [vp, dp, dp, dp, dp]
    lib.kks_set_wait_polls.argtypes = [vp, ctypes.c_int32]
    lib.kks_set_wait_polls.restype = ctypes.c_int
    lib.kks_bounds_report.argtypes = [ctypes.c_int, P(ctypes.c_int32), P(ctypes.c_uint64)]
    lib.kks_bounds_report.restype = ctypes.c_int
    lib.kks_elastic_fields.argtypes = [vp, dp, dp]
    lib.kks_checkpoint.argtypes = [vp, vp, ctypes.c_size_t, P(ctypes.c_size_t)]
    lib.kks_restore.argtypes = [vp, vp, ctypes.c_size_t]
    lib.kks_timing.argtypes = [vp, dp, P(ctypes.c_int64)]
    lib.kks_pipeline.argtypes = [vp, P(ctypes.c_int32), P(ctypes.c_int32)]
    lib.kks_adj_create.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int, P(vp)]
    lib.kks_adj_forward.argtypes = [vp, vp, dp, vp]
    lib.kks_adj_backward.argtypes = [vp, vp, vp, dp, vp, vp, dp]
    lib.kks_adj_destroy.argtypes = [vp]
    lib.kks_adj_set_precision.argtypes = [vp, ctypes.c_int]
    lib.kks_adj_backward_device.argtypes = [vp, vp, vp, dp, vp, vp, vp]
    lib.kks_adj_set_stream.argtypes = [vp, vp]
    for name in ("kks_adj_create", "kks_adj_forward", "kks_adj_backward", "kks_adj_destroy",
                 "kks_adj_set_precision", "kks_adj_backward_device", "kks_adj_set_stream"):
        getattr(lib, name).restype = ctypes.c_int
    lib.kks_destroy.argtypes = [vp]
    lib.kks_run_many.argtypes = [P(vp), ctypes.c_int32, P(ctypes.c_int32), P(ctypes.c_int32)]
    lib.kks_run_many.restype = ctypes.c_int
    lib.kks_batch_create.argtypes = [P(vp), ctypes.c_int32, ctypes.c_int32, P(vp)]
    lib.kks_batch_run.argtypes = [vp, P(ctypes.c_int32), P(ctypes.c_int32)]
    lib.kks_batch_timing.argtypes = [vp, dp, P(ctypes.c_int64)]
    lib.kks_batch_destroy.argtypes = [vp]
    lib.kks_get_launch_shape.argtypes = [vp, P(KksLaunchShape)]
    lib.kks_set_launch_shape.argtypes = [vp, P(KksLaunchShape)]
    lib.kks_autotune.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, P(KksLaunchShape), dp]
    for name in ("kks_batch_create", "kks_batch_run", "kks_batch_timing", "kks_batch_destroy",
                 "kks_get_launch_shape", "kks_set_launch_shape", "kks_autotune"):
        getattr(lib, name).restype = ctypes.c_int
    lib.kks_state_sums_noalloc.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, vp, vp]
    lib.kks_state_sums_noalloc.restype = ctypes.c_int
    i64p = P(ctypes.c_int64)
    lib.kks_voronoi_edges.argtypes = [vp, ctypes.c_int32, dp, i64p]
    lib.kks_generate_fields.argtypes = [vp, P(KksGenArgs)]
    lib.kks_place_precipitates.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int32, dp, dp, dp, dp]
    lib.kks_add_nuclei.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int32, dp, dp, dp, dp]
    lib.kks_count_below.argtypes = [vp, ctypes.c_double, i64p]
    lib.kks_insert_nuclei.argtypes = [vp, ctypes.c_double, ctypes.c_int32, i64p]
    for name in ("kks_voronoi_edges", "kks_generate_fields", "kks_place_precipitates", "kks_add_nuclei",
                 "kks_count_below", "kks_insert_nuclei"):
        getattr(lib, name).restype = ctypes.c_int
    lib.kks_last_error.restype = ctypes.c_char_p
    lib.kks_version.restype = ctypes.c_char_p
    for name in ("kks_create", "kks_upload", "kks_run", "kks_drain", "kks_get_state", "kks_download", "kks_download_pair",
                 "kks_elastic_fields", "kks_checkpoint", "kks_restore", "kks_timing", "kks_pipeline", "kks_destroy"):
        getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


class KksError(RuntimeError):
    """A C-ABI call returned an error code."""


def check(rc, what):
    if rc != KKS_OK:
        msg = load().kks_last_error().decode(errors="replace")
        raise KksError(f"{what} failed ({rc}): {msg}")


def bounds_report(device=0):
    """(checked, first): whether the loaded library is the bounds-check build,
    and the first out-of-range block it recorded on ``device`` since the last
    report (0 = none; site << 44 | index). Clears the record."""
    checked, first = ctypes.c_int32(0), ctypes.c_uint64(0)
    check(load().kks_bounds_report(int(device), ctypes.byref(checked), ctypes.byref(first)), "kks_bounds_report")
    return bool(checked.value), int(first.value)


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def as_field(a, n):
    """C-contiguous float64 copy-free view of a (nx, ny[, 1]) field."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.size != n:
        raise ValueError(f"field has {a.size} elements, expected {n}")
    return a
