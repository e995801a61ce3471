"""Simulation configuration (TOML), drop-in for ``pf_kks.config``.

``SimulationConfig`` carries exactly the fields of the reference dataclass
(``pf_kks/config.py:12-90``) with the same defaults, and ``load_config`` has the
same semantics (``pf_kks/config.py:93-108``): TOML sections are flattened,
keyword overrides that are not ``None`` win, unknown keys raise ``ValueError``.

The one addition is an optional ``[gpu]`` section, read into
``cfg.gpu`` (a :class:`GpuOptions`, kept out of ``to_dict`` so that the written
``config.json`` matches the reference's). ``fft_backend`` / ``fft_threads`` are
accepted and ignored: transforms always run on the GPU.
"""

import os
from dataclasses import asdict, dataclass, field, fields

import tomllib

PRECISIONS = ("fp64", "mixed", "mixed-cufft")


@dataclass
class GpuOptions:
    """Options of the GPU step (``[gpu]`` TOML section).

    precision : "fp64" (all-FP64 step, parity with the reference), "mixed"
        (FP32 transforms and pointwise math on the step increments with
        hand-written shared-memory FFTs; FP64 state, scalars, phase
        compositions and reductions) or "mixed-cufft" (the same step with
        cuFFT transforms).
    device : CUDA device ordinal.
    records_capacity : size of the device ring of per-attempt log records.
    autotune : before the run, give the cell the fastest launch shape
        (timed on the device on the initial state, then cached per GPU, grid
        and precision; pf_kks_gpu.autotune).
    """

    precision: str = "fp64"
    device: int = 0
    records_capacity: int = 1 << 15
    autotune: bool = False

    def __post_init__(self):
        if self.precision not in PRECISIONS:
            raise ValueError(f"unknown precision {self.precision!r}; expected one of {PRECISIONS}")


@dataclass
class SimulationConfig:
    # Grid (2-D: nz = 1). dy = dz = dx.
    nx: int = 735
    ny: int = 735
    nz: int = 1
    dx: float = 0.5e-9

    # Heat treatment: piecewise-linear temperature [K] vs time [s].
    schedule_time: list = field(default_factory=lambda: [0, 1350])
    schedule_temperature: list = field(default_factory=lambda: [400, 850])

    # Initial microstructure.
    precipitates: str = "../data/inputs/micro_final.npz"
    x_matrix: float = 0.025
    x_precipitate: float = 0.99999
    x_equilibrium: float = 0.025

    # Material data and calibration factors.
    material_tables: str = "../data/inputs/final_export.npz"
    c_gamma: float = 1.0
    c_eps0: float = 0.25
    c_D: float = 1.0
    c_Meta: float = 0.6
    D0: float | None = None
    QD: float | None = None
    Meta0: float = 5.60e-8
    QMeta: float = 1.10e5

    # Interface.
    alpha: float = 2.2
    half_width_cells: float = 2.5

    # Excess vacancies.
    T_quench: float = 850
    vacancy_sink_distance: float = 250e-9
    diffusion_enhancement_cap: float = 1e9

    # Time stepping (dimensionless time, unit dx^2 / D(t=0)).
    dtime_s: float = 75
    dtime_max: float = 400
    dtime_min_divisor: float = 1000
    residual_max: float = 1e-1
    residual_min: float = 1e-4
    step_factor: float = 1.25
    max_iterations: int = 50
    good_step_offset: int = 0

    # Run length and outputs.
    n_steps: int = 30000
    n_map_saves: int = 40
    n_surface_samples: int = 500
    surface_sample_last_step: int | None = None

    # FFT (accepted for compatibility; the GPU step always uses cuFFT).
    fft_backend: str = "auto"
    fft_threads: int = 12

    @property
    def dy(self):
        return 1 * self.dx

    @property
    def dz(self):
        return self.dx

    @property
    def lambd(self):
        return self.half_width_cells * self.dx

    @property
    def T_start(self):
        return self.schedule_temperature[0]

    def resolve_path(self, path, base):
        return path if os.path.isabs(path) else os.path.join(base, path)

    def to_dict(self):
        return asdict(self)

    @property
    def gpu_options(self):
        """The ``[gpu]`` options (defaults when the config was built in code)."""
        opts = self.__dict__.get("gpu")
        return opts if opts is not None else GpuOptions()


def load_config(path, **overrides):
    """Read a TOML configuration; keyword arguments override file values.

    Same behaviour as ``pf_kks.config.load_config`` for every reference key;
    the ``[gpu]`` section, if present, becomes ``cfg.gpu``.
    """
    with open(path, "rb") as f:
        data = tomllib.load(f)
    gpu = data.pop("gpu", None)
    flat = {}
    for key, value in data.items():
        if isinstance(value, dict):
            flat.update(value)
        else:
            flat[key] = value
    flat.update({k: v for k, v in overrides.items() if v is not None})
    known = {f.name for f in fields(SimulationConfig)}
    unknown = set(flat) - known
    if unknown:
        raise ValueError(f"unknown configuration keys: {sorted(unknown)}")
    cfg = SimulationConfig(**flat)
    if gpu is not None:
        gknown = {f.name for f in fields(GpuOptions)}
        gunknown = set(gpu) - gknown
        if gunknown:
            raise ValueError(f"unknown [gpu] configuration keys: {sorted(gunknown)}")
        cfg.gpu = GpuOptions(**gpu)
    return cfg
