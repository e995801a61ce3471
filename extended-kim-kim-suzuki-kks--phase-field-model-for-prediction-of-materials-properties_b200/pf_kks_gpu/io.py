"""Simulation maps (``.npz`` snapshots) and their file names.

The map is a data format shared with ``pf_kks.io`` (``pf_kks/io.py:20-40``):
the same ``.npz`` keys and dtypes and the same file name
``map{ttime:.2f}s_{T_start}_{T_max:.2f}K.npz``, so that maps written by either
implementation can be read by the other's tools.
"""

import os

import numpy as np

# Map keys, in the order they are written: the run time, six history lists
# up to the save step and the four fields (nx, ny, 1).
HISTORY_KEYS = (("time_out", "time"), ("T_out", "T"), ("X_al_mean_out", "X_al_mean"),
                ("X_th_mean_out", "X_th_mean"), ("eta_mean_out", "eta_mean"), ("surf_out", "surf"))
FIELD_KEYS = ("X", "X_al", "X_th", "eta")


def map_filename(ttime, T_start, T_max):
    """Map file name without extension: the run time and the maximum
    temperature with two decimals, the start temperature as Python prints it."""
    return f"map{ttime:.2f}s_{T_start}_{T_max:.2f}K"


def save_map(path, ttime, hist, X, X_al, X_th, eta):
    """Write one map: ``ttime``, the histories named in HISTORY_KEYS and the
    four fields, compressed."""
    arrays = {"ttime": ttime}
    arrays.update({key: hist[name] for key, name in HISTORY_KEYS})
    arrays.update(zip(FIELD_KEYS, (X, X_al, X_th, eta)))
    np.savez_compressed(path, **arrays)


def parse_map_filename(path):
    """(ttime, T_start, T_max) of a map file name; ValueError for any other
    name."""
    name = os.path.basename(path)
    try:
        if not (name.startswith("map") and name.endswith("K.npz")):
            raise ValueError
        ttime, rest = name[3:-5].split("s_", 1)
        T_start, T_max = rest.rsplit("_", 1)
        values = tuple(float(v) for v in (ttime, T_start, T_max))
    except ValueError:
        raise ValueError(f"not a map file name: {path}") from None
    if any(v < 0 for v in values):
        raise ValueError(f"not a map file name: {path}")
    return values
