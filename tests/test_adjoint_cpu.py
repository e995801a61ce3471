"""CPU checks of the differentiable fixed-dt step: the torch restatement of the
step (the autograd reference of the GPU adjoint) and the per-step coefficient
chain of pf_kks_gpu.adjoint, both against the oracle's unarmed attempts."""

import numpy as np
import pytest
import torch

from conftest import rel_l2, small_config
from kks_torch_step import TorchStep
from oracle import kks_oracle
from pf_kks_gpu import adjoint as A
from pf_kks_gpu import workloads
from pf_kks_gpu.generator import MicrostructureSpec
from pf_kks_gpu.materials import MaterialTables


def fixed_dt_case(nx=48, ny=40, n=6, seed=3):
    cfg = small_config(nx=nx, ny=ny, n_steps=n, x_equilibrium=0.0, n_map_saves=2, n_surface_samples=2)
    spec = MicrostructureSpec(nx, ny, n_cells=2, n_particles=8, r_min=3, r_max=6, seed=seed)
    state = workloads.initial_state(cfg, spec)
    tables = MaterialTables.from_npz(cfg.material_tables, cfg.c_gamma, cfg.c_eps0)
    return cfg, tables, state


def stepper_for(cfg, tables, device="cpu"):
    T0 = float(np.interp(0.0, cfg.schedule_time, cfg.schedule_temperature))
    return TorchStep(cfg.nx, cfg.ny, tables.at(T0, "C11"), tables.at(T0, "C12"), tables.at(T0, "C44"), device)


def as_tensor(state):
    nx, ny = state[0].shape[0], state[0].shape[1]
    return torch.tensor(np.stack([np.asarray(a, dtype=np.float64).reshape(nx, ny) for a in state]))


@pytest.mark.parametrize("n", [1, 6])
def test_torch_step_and_coefficients_match_oracle(n):
    cfg, tables, state = fixed_dt_case(n=n)
    ref = kks_oracle.run(cfg, *state, cfg.material_tables, write_logs=False, save_maps=False, max_steps=n)
    coef = A.coefficients(cfg, tables, n)
    step = stepper_for(cfg, tables)
    s = as_tensor(state)
    with torch.no_grad():
        for i in range(n):
            s = step(s, coef[i])
    for k, name in enumerate(("eta", "X", "X_al", "X_th")):
        assert rel_l2(s[k].numpy(), getattr(ref, name).reshape(cfg.nx, cfg.ny)) <= 1e-12, name
    # the temperatures the chain reaches are the oracle's
    assert ref.history["T"][-1] == pytest.approx(float(A._interp(
        torch.tensor(ref.history["time"][-1], dtype=torch.float64),
        torch.tensor(np.asarray(cfg.schedule_time, float)), torch.tensor(np.asarray(cfg.schedule_temperature,
                                                                                     float)))), rel=1e-14)


def test_coefficients_are_differentiable():
    cfg, tables, _ = fixed_dt_case(n=3)
    lcD = torch.zeros((), dtype=torch.float64, requires_grad=True)
    lcM = torch.zeros((), dtype=torch.float64, requires_grad=True)
    coef = A.coefficients(cfg, tables, 3, lcD, lcM)
    coef[:, 1].sum().backward()  # L_s depends on both D and Meta
    assert torch.isfinite(lcD.grad) and torch.isfinite(lcM.grad)
    assert float(lcM.grad) != 0.0


class _ToyEnthalpy:
    """Smooth stand-ins for the CALPHAD enthalpies (J/mol)."""

    def hm_fcc(self, T, x):
        return -2000.0 + 5.0 * T + 3.0e4 * x

    def hm_dia(self, T):
        return 1.0e4 + 2.0 * T

    def dhm_fcc_dx(self, T, x):
        return 3.0e4 + 0 * T + 0 * x


def test_finite_difference_dsc_follows_the_histories():
    cfg, tables, _ = fixed_dt_case(n=5)
    coef, t, T = A.coefficients(cfg, tables, 5, return_times=True)
    assert t[0] == 0 and torch.all(t[1:] > t[:-1])
    assert float(T[-1]) == pytest.approx(float(np.interp(float(t[-1]), cfg.schedule_time, cfg.schedule_temperature)))
    f = torch.tensor([0.10, 0.11, 0.13, 0.16, 0.17], dtype=torch.float64, requires_grad=True)
    x = torch.tensor([0.020, 0.019, 0.017, 0.016, 0.0158], dtype=torch.float64, requires_grad=True)
    q = A.finite_difference_dsc(f, x, t, T, _ToyEnthalpy(), heating_rate=20 / 60)
    assert q.shape == (4,)
    # by hand for the first interval
    e = _ToyEnthalpy()
    dt0 = float(t[1] - t[0])
    T0 = float(T[0])
    ref0 = ((1 - 0.10) * 3.0e4 * (0.019 - 0.020) / dt0 / A.M_AL
            + (0.11 - 0.10) / dt0 * (e.hm_dia(T0) / A.M_SI - e.hm_fcc(T0, 0.020) / A.M_AL)) / (20 / 60)
    assert float(q[0].detach()) == pytest.approx(ref0, rel=1e-12)
    q.sum().backward()
    assert torch.all(torch.isfinite(f.grad)) and torch.all(torch.isfinite(x.grad))
