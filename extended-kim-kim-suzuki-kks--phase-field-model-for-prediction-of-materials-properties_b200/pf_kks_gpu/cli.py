"""``pf-kks-run`` on the GPU: the reference's command line (``pf_kks/cli.py:25-56``).

The interface is the reference's: a TOML configuration, ``--out``,
``--n-steps``, ``--fft-threads`` (accepted, unused: the transforms are on the
GPU), ``--print-config`` and ``--quiet``; the output directory receives
``config.json``, ``saved_maps/map*.npz``, ``log.txt``, ``dtime.txt`` and
``history.npz`` in the reference's formats. Added options: ``--precision``,
``--device`` and ``--autotune`` (their defaults come from the ``[gpu]``
section of the configuration).

The initial state is the reference CLI's: sharp precipitates read from the
configuration's ``precipitates`` file, placed in a uniform matrix. Paths in
the configuration are relative to the configuration file's directory.

    pf-kks-run CONFIG --out DIR [--n-steps N] [--precision mixed]
    python -m pf_kks_gpu.cli CONFIG --out DIR ...
"""

import argparse
import json
import os
import sys
from pathlib import Path

import numpy as np

from . import solver
from .config import load_config
from .microstructure import load_precipitates, place_precipitates

# (flags, keyword arguments of add_argument): the reference's options first.
OPTIONS = (
    (("config",), dict(help="simulation configuration (TOML)")),
    (("--out",), dict(default="outputs/run", help="directory for maps, logs and histories (default: %(default)s)")),
    (("--n-steps",), dict(type=int, help="run this many steps instead of the configured n_steps")),
    (("--fft-threads",), dict(type=int, help="kept for configuration compatibility; the GPU step ignores it")),
    (("--print-config",), dict(action="store_true", help="print the resolved configuration as JSON and stop")),
    (("--quiet",), dict(action="store_true", help="no progress output")),
    (("--precision",), dict(choices=("fp64", "mixed", "mixed-cufft"), help="precision of the GPU step")),
    (("--device",), dict(type=int, help="CUDA device ordinal")),
    (("--autotune",), dict(action="store_true", help="time the launch shapes on the initial state first")),
)


def build_parser():
    parser = argparse.ArgumentParser(
        prog="pf-kks-run",
        description="Extended-KKS phase-field run on one GPU. Writes config.json, saved_maps/, log.txt, "
                    "dtime.txt and history.npz into --out; data paths in CONFIG are relative to its directory.")
    for flags, kwargs in OPTIONS:
        parser.add_argument(*flags, **kwargs)
    return parser


def write_history(path, result):
    """history.npz: every history list, ``good_step`` (-1 when the adaptive
    scheme never armed) and ``ttime``."""
    arrays = {name: np.asarray(values) for name, values in result.history.items()}
    good = -1 if result.good_step is None else result.good_step
    np.savez_compressed(path, good_step=good, ttime=result.ttime, **arrays)


def main(argv=None):
    args = build_parser().parse_args(argv)
    cfg = load_config(args.config, n_steps=args.n_steps, fft_threads=args.fft_threads)
    resolved = cfg.to_dict()
    if args.print_config:
        print(json.dumps(resolved, indent=2))
        return 0

    if args.autotune:
        options = cfg.gpu_options
        options.autotune = True
        cfg.gpu = options
    base_dir = str(Path(args.config).resolve().parent)
    out = args.out
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(out, "config.json"), "w") as f:
        json.dump(resolved, f, indent=2)

    circles = load_precipitates(cfg.resolve_path(cfg.precipitates, base_dir))  # ox, oy, oz, r
    state = place_precipitates(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz, cfg.x_matrix, cfg.x_precipitate,
                               circles[3], *circles[:3])
    result = solver.run(cfg, *state, out_dir=out, base_dir=base_dir, verbose=not args.quiet,
                        precision=args.precision, device=args.device)
    write_history(os.path.join(out, "history.npz"), result)
    return 0


def entry():
    """Console-script entry (``pf-kks-run``)."""
    sys.exit(main())


if __name__ == "__main__":
    entry()
