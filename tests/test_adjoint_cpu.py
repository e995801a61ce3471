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


def test_thermo_restatement_matches_reference():
    """The torch restatement of the CALPHAD functions of the simulated DSC
    against pf_kks.thermo (golden/make_thermo_fixture.py)."""
    from conftest import GOLDEN
    from pf_kks_gpu import dsc

    g = np.load(f"{GOLDEN}/reference_thermo.npz")
    T = torch.tensor(g["T"])[:, None].expand(-1, g["x"].size)
    x = torch.tensor(g["x"])[None, :].expand(g["T"].size, -1)
    th = dsc.phase_thermo(T, x)
    for name, value in (("Hm_fcc", th.Hm_fcc), ("d_Hm_fcc_dSi", th.dHm_fcc_dx), ("cp_fcc", th.cp_fcc),
                        ("Vmfcc", th.Vm_fcc)):
        np.testing.assert_allclose(value.numpy(), g[name], rtol=1e-12, atol=0, err_msg=name)
    for name, value in (("Hm_dia", th.Hm_dia[:, 0]), ("cp_dia", th.cp_dia[:, 0]), ("Vmdia", th.Vm_dia[:, 0])):
        np.testing.assert_allclose(value.numpy(), g[name], rtol=1e-12, atol=0, err_msg=name)


def test_thermo_derivative_in_x_is_the_enthalpy_slope():
    from pf_kks_gpu import dsc

    T = torch.tensor([450.0, 520.0, 710.0], dtype=torch.float64)
    x = torch.tensor([0.004, 0.02, 0.05], dtype=torch.float64, requires_grad=True)
    th = dsc.phase_thermo(T, x)
    (g,) = torch.autograd.grad(th.Hm_fcc.sum(), x)
    np.testing.assert_allclose(g.numpy(), th.dHm_fcc_dx.detach().numpy(), rtol=1e-12)


def test_simulated_dsc_terms_by_hand():
    """The three terms of pf_kks/postprocess/dsc.py:121-130 with forward
    differences, checked by hand on the first interval."""
    from pf_kks_gpu import dsc

    cfg, tables, _ = fixed_dt_case(n=5)
    coef, t, T = A.coefficients(cfg, tables, 5, return_times=True)
    assert t[0] == 0 and torch.all(t[1:] > t[:-1])
    assert float(T[-1]) == pytest.approx(float(np.interp(float(t[-1]), cfg.schedule_time, cfg.schedule_temperature)))
    f = torch.tensor([0.10, 0.11, 0.13, 0.16, 0.17], dtype=torch.float64, requires_grad=True)
    x = torch.tensor([0.020, 0.019, 0.017, 0.016, 0.0158], dtype=torch.float64, requires_grad=True)
    surf = torch.tensor([1.0e-8, 1.2e-8, 1.1e-8, 1.5e-8, 1.6e-8], dtype=torch.float64)
    p = dsc.DSCParameters.for_config(cfg)
    q = dsc.simulated_dsc(f, x, surf, t, T, p)
    assert q.total.shape == (4,)
    dt0, T0 = float(t[1] - t[0]), float(T[0])
    th = dsc.phase_thermo(torch.tensor([T0], dtype=torch.float64), torch.tensor([0.020], dtype=torch.float64))
    rho = 0.10 * dsc.M_SI / float(th.Vm_dia) + 0.90 * dsc.M_AL / float(th.Vm_fcc)
    bg = p.heating_rate * (0.10 * float(th.cp_dia) / dsc.M_SI + 0.90 * float(th.cp_fcc) / dsc.M_AL)
    su = p.interface_energy * (0.2e-8) / dt0 / (p.simulated_area * rho)
    pr = (0.90 * float(th.dHm_fcc_dx) / dsc.M_AL * (0.019 - 0.020) / dt0
          + (0.11 - 0.10) / dt0 * (float(th.Hm_dia) / dsc.M_SI - float(th.Hm_fcc) / dsc.M_AL))
    assert float(q.background[0]) == pytest.approx(bg, rel=1e-12)
    assert float(q.surface[0]) == pytest.approx(su, rel=1e-12)
    assert float(q.precipitation[0]) == pytest.approx(pr, rel=1e-12)
    assert float(q.total[0]) == pytest.approx((bg + su + pr) * p.output_scale, rel=1e-12)
    q.total.sum().backward()
    assert torch.all(torch.isfinite(f.grad)) and torch.all(torch.isfinite(x.grad))


def test_three_parameter_offsets():
    """c_gamma scales the interface energy: kappa^2 and w scale with it, while
    the thin-interface L (pf_kks/kinetics.py:72-80) does not depend on it
    (sigma / kappa^2 and kappa / sqrt(w) are both free of sigma). The
    annealing-rate offset moves the vacancy fraction and with it D. Zero
    offsets reproduce the unperturbed chain bit for bit."""
    cfg, tables, _ = fixed_dt_case(n=4)
    base = A.coefficients(cfg, tables, 4)
    z = torch.zeros((), dtype=torch.float64)
    same = A.coefficients(cfg, tables, 4, z, z, log_c_gamma=z, log_anneal=z)
    assert torch.equal(base, same)
    lg = torch.tensor(np.log(1.1), dtype=torch.float64)
    g = A.coefficients(cfg, tables, 4, log_c_gamma=lg)
    np.testing.assert_allclose((g[:, 2] / base[:, 2]).numpy(), 1.1, rtol=1e-14)  # kappa^2 ~ gamma
    np.testing.assert_allclose((g[:, 4] / base[:, 4]).numpy(), 1.1, rtol=1e-14)  # w ~ gamma
    np.testing.assert_allclose(g[:, 1].numpy(), base[:, 1].numpy(), rtol=1e-14)
    la = torch.tensor(np.log(0.8), dtype=torch.float64, requires_grad=True)
    an = A.coefficients(cfg, tables, 4, log_anneal=la)
    an[1:, 3].sum().backward()  # D_s of the steps after the first relaxation
    assert float(la.grad) != 0.0
