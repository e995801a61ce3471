"""Command-line entry point, drop-in for ``pf-kks-run`` (``pf_kks/cli.py:25-56``).

Same arguments and outputs: ``saved_maps/map*.npz``, ``history.npz``,
``log.txt``, ``dtime.txt`` and ``config.json`` in ``--out``. Additions:
``--precision {fp64,mixed}``, ``--device N`` and ``--autotune`` (else taken
from the ``[gpu]`` section of the configuration).

Usage: python -m pf_kks_gpu.cli CONFIG --out DIR [--n-steps N] [--precision mixed]
"""

import argparse
import json
import os
from pathlib import Path

import numpy as np

from . import solver
from .config import load_config
from .microstructure import load_precipitates, place_precipitates

DESCRIPTION = """Run a phase-field simulation on the GPU from a TOML configuration.

Relative data paths in the configuration are resolved against the directory of
the configuration file.

Outputs (in --out): saved_maps/map*.npz snapshots, history.npz (per-step
histories and residuals), log.txt, dtime.txt and config.json (the resolved
configuration).
"""


def main(argv=None):
    parser = argparse.ArgumentParser(description=DESCRIPTION, formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("config", help="TOML configuration file")
    parser.add_argument("--out", default="outputs/run", help="output directory (default: outputs/run)")
    parser.add_argument("--n-steps", type=int, help="override the number of steps")
    parser.add_argument("--fft-threads", type=int, help="accepted for compatibility (ignored: cuFFT)")
    parser.add_argument("--print-config", action="store_true", help="print the resolved configuration and exit")
    parser.add_argument("--quiet", action="store_true", help="do not print progress")
    parser.add_argument("--precision", choices=("fp64", "mixed"), help="GPU step precision")
    parser.add_argument("--device", type=int, help="CUDA device ordinal")
    parser.add_argument("--autotune", action="store_true",
                        help="time the launch shapes on the initial state first (cached per GPU and grid)")
    args = parser.parse_args(argv)

    cfg = load_config(args.config, n_steps=args.n_steps, fft_threads=args.fft_threads)
    base_dir = str(Path(args.config).resolve().parent)
    if args.print_config:
        print(json.dumps(cfg.to_dict(), indent=2))
        return 0

    if args.autotune:
        opts = cfg.gpu_options
        opts.autotune = True
        cfg.gpu = opts
    os.makedirs(args.out, exist_ok=True)
    with open(os.path.join(args.out, "config.json"), "w") as f:
        json.dump(cfg.to_dict(), f, indent=2)

    ox, oy, oz, r = load_precipitates(cfg.resolve_path(cfg.precipitates, base_dir))
    state = place_precipitates(
        cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz, cfg.x_matrix, cfg.x_precipitate, r, ox, oy, oz
    )
    result = solver.run(cfg, *state, out_dir=args.out, base_dir=base_dir, verbose=not args.quiet,
                        precision=args.precision, device=args.device)
    np.savez_compressed(
        os.path.join(args.out, "history.npz"),
        good_step=-1 if result.good_step is None else result.good_step,
        ttime=result.ttime,
        **{k: np.asarray(v) for k, v in result.history.items()},
    )
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
