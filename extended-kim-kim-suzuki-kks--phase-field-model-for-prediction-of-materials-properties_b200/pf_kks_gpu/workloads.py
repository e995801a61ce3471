"""The measured workloads: configurations plus seeded initial states.

Each workload is a :class:`SimulationConfig` (the demo_small /
reproducible_run parameter set of the reference, ``configs/demo_small.toml``)
and a generator specification (:mod:`pf_kks_gpu.generator`). Vacancies start
at a site fraction of 1e-4 through the existing ``T_quench`` key:
``quenched_vacancy_fraction(816.3448 K) = 1e-4``. Runs that only need the
final state use ``n_map_saves = 2`` (maps at step 1 and at the end): the run
length is the last map step (``pf_kks/solver.py:48-53``), so a single map
save would stop the run after its first step.

=========  ==========================================================================
name       setup
=========  ==========================================================================
demo160    160^2, 4 Voronoi cells, ~40 particles R~U(3,8); 400->850 K at 20 K/min
           (schedule [0,1350] s), 2000 adaptive steps, FP64
iso735     735^2, 20 cells, ~300 particles; isothermal 500 K, 500 fixed-dt steps
           (x_equilibrium = 0 never arms the adaptive scheme)
ramp1420   1420^2, 40 cells, ~1200 particles R~U(3,10); 400->719 K at 20 K/min,
           adaptive, mixed precision
ensemble   48 cells of side {128,192,256,384,512}, seeds 0-47, particles
           proportional to area, heating U(5,40) K/min from 400 to 600 K
adjoint256 256^2, 8 cells; 500->520 K ramp, 300 fixed-dt steps at the demo parameters; the
           target DSC comes from the same run with Si mobility x 1.2, vacancy annealing
           rate x 0.8 and interface energy x 1.1 (ADJOINT_TARGET_FACTORS)
=========  ==========================================================================
"""

import numpy as np

from .config import GpuOptions, SimulationConfig
from .generator import MicrostructureSpec, generate, generate_on_device
from .materials import DEFAULT_TABLES, MaterialTables

T_QUENCH_XV_1E4 = 816.3448


def base_config(**kw):
    p = dict(
        nx=160,
        ny=160,
        dx=0.5e-9,
        schedule_time=[0, 1350],
        schedule_temperature=[400, 850],
        material_tables=DEFAULT_TABLES,
        c_eps0=0.25,
        c_Meta=0.6,
        T_quench=T_QUENCH_XV_1E4,
        n_steps=2000,
        n_map_saves=10,
        n_surface_samples=100,
    )
    p.update(kw)
    return SimulationConfig(**p)


def heating_schedule(T0, T1, rate_K_per_min):
    return [0, (T1 - T0) * 60.0 / rate_K_per_min], [T0, T1]


def initial_state(cfg, spec):
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    T0 = np.interp(0, np.array(cfg.schedule_time), np.array(cfg.schedule_temperature))
    return generate(spec, *(tables.at(T0, n) for n in ("A_alp", "B_alp", "A_thet", "B_thet")))


def demo160(n_steps=2000, precision="fp64", seed=0):
    cfg = base_config(nx=160, ny=160, n_steps=n_steps)
    cfg.gpu = GpuOptions(precision=precision)
    spec = MicrostructureSpec(160, 160, n_cells=4, n_particles=40, r_min=3, r_max=8, seed=seed)
    return cfg, spec


def iso735(n_steps=500, precision="fp64", seed=0):
    cfg = base_config(nx=735, ny=735, n_steps=n_steps, schedule_time=[0, 1], schedule_temperature=[500, 500],
                      x_equilibrium=0.0, n_map_saves=2, n_surface_samples=50)
    cfg.gpu = GpuOptions(precision=precision)
    spec = MicrostructureSpec(735, 735, n_cells=20, n_particles=300, r_min=3, r_max=8, seed=seed)
    return cfg, spec


def ramp1420(n_steps=30000, precision="mixed", seed=0):
    t, T = heating_schedule(400.0, 719.0, 20.0)
    cfg = base_config(nx=1420, ny=1420, n_steps=n_steps, schedule_time=t, schedule_temperature=T, n_map_saves=2,
                      n_surface_samples=min(500, n_steps))
    cfg.gpu = GpuOptions(precision=precision)
    spec = MicrostructureSpec(1420, 1420, n_cells=40, n_particles=1200, r_min=3, r_max=10, seed=seed)
    return cfg, spec


ENSEMBLE_SIDES = (128, 192, 256, 384, 512)


def ensemble(n_instances=48, n_steps=1000, precision="mixed"):
    """Per-instance (cfg, spec) list: side, seed and heating rate drawn from a
    generator seeded with 2024 (sides uniform in ENSEMBLE_SIDES, rate U(5,40)
    K/min, 400 -> 600 K)."""
    rng = np.random.Generator(np.random.PCG64(2024))
    sides = rng.choice(np.array(ENSEMBLE_SIDES), size=n_instances)
    rates = rng.uniform(5.0, 40.0, size=n_instances)
    out = []
    for i in range(n_instances):
        n = int(sides[i])
        t, T = heating_schedule(400.0, 600.0, float(rates[i]))
        cfg = base_config(nx=n, ny=n, n_steps=n_steps, schedule_time=t, schedule_temperature=T, n_map_saves=2,
                          n_surface_samples=min(100, n_steps))
        cfg.gpu = GpuOptions(precision=precision)
        n_part = max(1, int(round(40 * (n / 160.0) ** 2)))
        spec = MicrostructureSpec(n, n, n_cells=max(1, int(round(4 * (n / 160.0) ** 2))), n_particles=n_part,
                                  r_min=3, r_max=8, seed=i)
        out.append((cfg, spec))
    return out


# (Si mobility prefactor, vacancy annealing rate, interface energy) of the
# target run of the gradient workload, relative to the base parameters
ADJOINT_TARGET_FACTORS = (1.2, 0.8, 1.1)


def adjoint256(n_steps=300, precision="fp64", seed=0, factors=(1.0, 1.0, 1.0)):
    """Fixed-dt run for gradients at the demo parameters; ``factors``
    multiply the Si mobility prefactor (c_D), the vacancy annealing rate
    (Deff / Lv^2: the sink distance is divided by its square root) and the
    interface energy (c_gamma)."""
    fD, fA, fG = factors
    cfg = base_config(nx=256, ny=256, n_steps=n_steps, schedule_time=[0, 60.0], schedule_temperature=[500, 520],
                      x_equilibrium=0.0, n_map_saves=2, n_surface_samples=n_steps, c_D=1.0 * fD,
                      vacancy_sink_distance=250e-9 / fA**0.5, c_gamma=1.0 * fG)
    cfg.gpu = GpuOptions(precision=precision)
    spec = MicrostructureSpec(256, 256, n_cells=8, n_particles=102, r_min=3, r_max=8, seed=seed)
    return cfg, spec


def initial_state_on_device(cell, cfg, spec):
    """``initial_state`` written by the device straight into ``cell``."""
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    T0 = np.interp(0, np.array(cfg.schedule_time), np.array(cfg.schedule_temperature))
    return generate_on_device(cell, spec, *(tables.at(T0, n) for n in ("A_alp", "B_alp", "A_thet", "B_thet")))
