"""Launch-shape autotuner with an on-disk cache.

A cell's attempt has three launch choices (``kks_launch_shape``): for the mixed
precision, the fused shared-memory FFT passes or the cuFFT passes; the number
of y-frequency columns a fused column-pass block transforms (1..4: more
columns mean fewer, larger blocks and more prime-stage work per barrier); and
the grid of the grid-stride field kernels. ``kks_autotune`` times every
candidate on the cell's own state on the device (CUDA events, the state saved
before and restored after) and keeps the fastest. The choice depends on the
GPU, the grid and the precision only, so it is cached per
``(device name, nx, ny, precision)`` in a JSON file and re-applied to later
cells of the same key without timing again.

The cache file is ``$KKS_AUTOTUNE_CACHE``, else
``~/.cache/pf_kks_gpu/launch_shapes.json``.
"""

import json
import os


def cache_path():
    return os.environ.get("KKS_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "pf_kks_gpu", "launch_shapes.json"))


def device_name(device=0):
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:
        return f"cuda:{device}"


def key(cell, device=0, batchable=False):
    return f"{device_name(device)}|{cell.nx}x{cell.ny}|{cell.precision}" + ("|batch" if batchable else "")


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune(cell, attempts=20, device=0, cache=True, force=False, batchable=False):
    """Give ``cell`` its fastest launch shape. With ``cache``, a shape stored
    for the cell's key is applied without timing (unless ``force``); a new
    measurement is stored. ``batchable``: only shapes with which the cell can
    join a batch. Returns {"shape", "ms_per_attempt", "source"}."""
    path = cache_path()
    k = key(cell, device, batchable)
    table = _load(path) if cache else {}
    if cache and not force and k in table:
        shape = table[k]["shape"]
        cell.set_launch_shape(shape["pipeline"], shape["cols"], shape["field_blocks"])
        return {"shape": shape, "ms_per_attempt": table[k]["ms_per_attempt"], "source": "cache"}
    shape, ms = cell.autotune(attempts, batchable=batchable)
    if cache:
        table = _load(path)
        table[k] = {"shape": shape, "ms_per_attempt": ms}
        try:
            _store(path, table)
        except OSError:
            pass  # a read-only home: the tuned shape still applies to this cell
    return {"shape": shape, "ms_per_attempt": ms, "source": "measured"}
