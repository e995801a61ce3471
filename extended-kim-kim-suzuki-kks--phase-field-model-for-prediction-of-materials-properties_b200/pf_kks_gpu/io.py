"""Simulation maps (``.npz`` snapshots) and their file names.

Byte-compatible with ``pf_kks.io`` (``pf_kks/io.py:20-62``): same keys, dtypes
and ``map{ttime:.2f}s_{T_start}_{T_max:.2f}K.npz`` names, so maps written by
either implementation can be read by the other's tools.
"""

import glob
import os
import re

import numpy as np

MAP_PATTERN = re.compile(r"map(?P<ttime>[0-9.]+)s_(?P<T_start>[0-9.]+)_(?P<T_max>[0-9.]+)K\.npz$")


def map_filename(ttime, T_start, T_max):
    """Map file name without extension (pf_kks/io.py:20-22)."""
    return "map" + "{0:.2f}".format(ttime) + "s_" + str(T_start) + "_" + "{0:.2f}".format(T_max) + "K"


def save_map(path, ttime, hist, X, X_al, X_th, eta):
    """Write a map (pf_kks/io.py:25-40)."""
    np.savez_compressed(
        path,
        ttime=ttime,
        time_out=hist["time"],
        T_out=hist["T"],
        X_al_mean_out=hist["X_al_mean"],
        X_th_mean_out=hist["X_th_mean"],
        eta_mean_out=hist["eta_mean"],
        surf_out=hist["surf"],
        X=X,
        X_al=X_al,
        X_th=X_th,
        eta=eta,
    )


def parse_map_filename(path):
    m = MAP_PATTERN.search(os.path.basename(path))
    if m is None:
        raise ValueError(f"not a map file name: {path}")
    return float(m["ttime"]), float(m["T_start"]), float(m["T_max"])


def list_maps(directory):
    files = [f for f in glob.glob(os.path.join(directory, "map*.npz")) if MAP_PATTERN.search(os.path.basename(f))]
    return sorted(files, key=lambda f: (parse_map_filename(f)[2], parse_map_filename(f)[0]))


def load_map(path, fields=True):
    with np.load(path) as d:
        keys = d.files if fields else [k for k in d.files if k not in ("X", "X_al", "X_th", "eta")]
        return {k: d[k] for k in keys}
