"""pf_kks_gpu: the semi-implicit extended-KKS phase-field step on a B200.

Drop-in for the solver path of the reference package ``pf_kks``: the same
``SimulationConfig`` / ``load_config`` (TOML), ``solver.run`` signature,
``SimulationResult``, ``AdaptiveStepError``, saved maps, ``history.npz`` and
run logs, with every attempt of the time step running in hand-written sm_100a
CUDA kernels and cuFFT behind the C ABI of ``include/kks.h``.
"""

__version__ = "1.0.0"
