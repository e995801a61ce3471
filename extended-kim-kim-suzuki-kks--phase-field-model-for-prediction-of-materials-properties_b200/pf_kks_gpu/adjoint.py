"""Gradients of history functionals (a simulated DSC, for instance) of a
fixed-dt run with respect to the kinetic parameters.

A fixed-dt run is the attempt loop of ``pf_kks.solver.run`` before the
adaptive scheme arms (``pf_kks/solver.py:176-290`` with ``flag == 0``; set
``x_equilibrium = 0`` to keep it unarmed): every step is one attempt, and its
coefficients depend only on the heat-treatment schedule and the kinetic
parameters, not on the fields. The gradient is therefore split in two:

* :func:`coefficients` restates the per-attempt scalar chain of the reference
  (schedule T(t), vacancy relaxation, Si diffusivity, interface mobility,
  Allen-Cahn coefficient, normalisation; ``pf_kks/kinetics.py:9-107``,
  ``pf_kks/solver.py:179-240``) in float64 torch, so that the 15 per-step
  coefficients are differentiable functions of log-scale offsets of four
  parameters: the Si mobility prefactor ``c_D`` (``D0``), the interface
  mobility ``c_Meta``, the interface energy ``c_gamma`` (the gamma table,
  ``pf_kks/materials.py:50-51``: it enters kappa^2, w and L) and the vacancy
  annealing rate (``Deff / Lv^2``, ``pf_kks/kinetics.py:52-56``: the offset
  divides ``vacancy_sink_distance^2``).
* :class:`FixedDtRun` runs the field steps on the GPU (``kks_adj_forward``)
  and, in its backward pass, the hand-written adjoint of the step
  (``kks_adj_backward``, ``csrc/kks_adjoint.cu``), checkpointing the state
  every ``checkpoint_every`` steps and recomputing the steps in between. It
  returns the per-step histories ``eta_mean`` and ``X_al_mean`` of the
  reference (``pf_kks/solver.py:380-390``: mean of eta, mean of X over
  eta < 0.05, both of the step's input state), the interface measure ``surf``
  of each step's input state (a cell count: no gradient) and the final state.

:func:`dsc_of_run` chains both with the simulated DSC of :mod:`pf_kks_gpu.dsc`.
The window is fixed in steps, as the reference's API counts it: a change of
``c_D`` changes D(t = 0) and with it the physical time of every step
(``dx^2 / D_0 * dtime_s``, ``pf_kks/solver.py:188-190, 368-369``), so the
times and temperatures of the steps are differentiable outputs too.

    theta = torch.zeros(3, dtype=torch.float64, requires_grad=True)  # log c_D, log rate, log c_gamma
    q = dsc_of_run(cfg, tables, state0, stepper, n_steps, theta, checkpoint_every=50).total
    loss = ((q - q_target) ** 2).sum(); loss.backward()               # -> theta.grad
"""

import ctypes

import numpy as np

from . import _lib as L
from .kinetics import quenched_vacancy_fraction

# constants of pf_kks/constants.py:6-21
_R = 8.314472
_HF1VA, _SF1VA, _HB, _SB_KB, _Z = 63680, 2.49, 10613, 42453, 12
_D0_AL, _Q_AL, _D0_SI, _Q_SI = 1.7e-4, 142e3, 3.66e-6, 110958


def _torch():
    import torch

    return torch


def _interp(x, xp, fp):
    """np.interp at a scalar tensor x (end values outside the table); the
    result is differentiable in x and fp."""
    torch = _torch()
    n = xp.numel()
    if n == 1:
        return fp[0] + 0 * x
    xd = float(x.detach())
    if xd <= float(xp[0]):
        return fp[0] + 0 * x
    if xd >= float(xp[-1]):
        return fp[-1] + 0 * x
    i = int(torch.searchsorted(xp, torch.tensor([xd], dtype=xp.dtype), right=True)[0]) - 1
    slope = (fp[i + 1] - fp[i]) / (xp[i + 1] - xp[i])
    return slope * (x - xp[i]) + fp[i]


def coefficients(cfg, tables, n_steps, log_c_D=None, log_c_Meta=None, return_times=False, log_c_gamma=None,
                 log_anneal=None):
    """Per-step coefficients of a fixed-dt run, shape (n_steps, 15), float64,
    in the order of ``KKS_COEF_*`` (``include/kks.h``).

    The log offsets (0-d float64 tensors, default 0; gradients flow to them)
    multiply ``cfg.c_D`` (``log_c_D``), ``cfg.c_Meta`` (``log_c_Meta``), the
    interface energy of the tables (``log_c_gamma``, on top of ``cfg.c_gamma``)
    and the vacancy annealing rate Deff / Lv^2 (``log_anneal``) by their
    exponential. With ``return_times`` the result is (coef, time, T): the time
    [s] and temperature [K] of each step's input state (the ``time`` / ``T``
    histories), which also depend on the parameters through D(t = 0).
    """
    torch = _torch()
    f64 = torch.float64
    zero = torch.zeros((), dtype=f64)
    lcD = zero if log_c_D is None else log_c_D
    lcM = zero if log_c_Meta is None else log_c_Meta
    lcG = zero if log_c_gamma is None else log_c_gamma
    lAn = zero if log_anneal is None else log_anneal
    D0 = float(tables.D0 if cfg.D0 is None else cfg.D0) * cfg.c_D * torch.exp(lcD)
    QD = float(tables.QD if cfg.QD is None else cfg.QD)
    Meta0 = cfg.Meta0 * cfg.c_Meta * torch.exp(lcM)
    QMeta = float(cfg.QMeta)
    Lv2 = cfg.vacancy_sink_distance**2 / torch.exp(lAn)
    lambd = cfg.half_width_cells * cfg.dx
    dx = cfg.dx
    cap = cfg.diffusion_enhancement_cap
    st = torch.tensor(np.asarray(cfg.schedule_time, dtype=np.float64), dtype=f64)
    sT = torch.tensor(np.asarray(cfg.schedule_temperature, dtype=np.float64), dtype=f64)
    tT = torch.tensor(np.asarray(tables.T, dtype=np.float64), dtype=f64)
    tab = {name: torch.tensor(np.asarray(getattr(tables, name), dtype=np.float64), dtype=f64)
           for name in ("A_alp", "B_alp", "C_alp", "A_thet", "B_thet", "C_thet", "C44", "epsX", "Vm", "gamma",
                        "X_Si_fcc")}
    dtime_s_ini = float(cfg.dtime_s)
    dtime_s_min = dtime_s_ini / cfg.dtime_min_divisor
    dtime_s = dtime_s_ini  # clamped like the prologue does (pf_kks/solver.py:198-201)
    if dtime_s > cfg.dtime_max:
        dtime_s = cfg.dtime_max
    if dtime_s < dtime_s_min:
        dtime_s = dtime_s_min
    Xv = torch.tensor(float(quenched_vacancy_fraction(cfg.T_quench)), dtype=f64)
    t = zero
    rows, times, temps = [], [], []
    D_0 = None
    for n in range(n_steps):
        T = _interp(t, st, sT)
        times.append(t)
        temps.append(T)
        Xve = torch.exp(-(_HF1VA - T * _SF1VA) / (_R * T)) * (1 - _Z * 0.01 + _Z * 0.01 * torch.exp(
            (_HB - T * _SB_KB) / (_R * T)))
        factor = torch.abs(1 + (Xv - Xve) / Xve)
        arr = torch.exp(-QD / (_R * T))
        D = torch.where(factor > cap, cap * D0 * arr, factor * D0 * arr)
        D = torch.where(factor < 1, D0 * arr, D)
        Meta = Meta0 * torch.exp(-QMeta / (_R * T))
        Deff = torch.abs(1 + (Xv - Xve) / Xve) * (0.03 * _D0_SI * torch.exp(-_Q_SI / (_R * T)) +
                                                  0.97 * _D0_AL * torch.exp(-_Q_AL / (_R * T)))
        if n == 0:
            D_0 = D
        dtime = (dx**2 / D_0) * dtime_s_ini
        Xv = Xv + (1 - torch.exp(-dtime * (Deff / Lv2))) * (Xve - Xv)
        at = {k: _interp(T, tT, v) for k, v in tab.items()}
        sigma, Omega0 = at["gamma"] * torch.exp(lcG), at["Vm"]
        kappa2 = 2 * lambd * sigma * 3 / cfg.alpha
        w = (sigma * 3 * cfg.alpha) / lambd
        kappa = torch.sqrt(kappa2)
        xi = (19 / 30) * (1 / Omega0) * 2 * at["A_alp"] * (at["X_Si_fcc"] - 0.9999) ** 2
        Lc = (sigma / kappa**2) * (1 / (1 / Meta + kappa * xi / (D * torch.sqrt(2 * w)))) * 0.01
        C44 = at["C44"]
        s = C44 * Omega0
        rows.append(torch.stack([
            torch.tensor(dtime_s, dtype=f64), (Lc * C44 * dx**2) / D_0, kappa2 / (C44 * dx**2), D / D_0, w / C44,
            at["A_alp"] / s, at["B_alp"] / s, at["C_alp"] / s, at["A_thet"] / s, at["B_thet"] / s, at["C_thet"] / s,
            at["epsX"], C44, (at["B_alp"] - at["B_thet"]) / (2 * at["A_thet"]), at["A_alp"] / at["A_thet"]]))
        t = t + (dx**2 / D_0) * dtime_s
    if return_times:
        return torch.stack(rows), torch.stack(times), torch.stack(temps)
    return torch.stack(rows)


class StepAdjoint:
    """The fixed-dt step and its adjoint on one GPU (a ``kks_adj`` handle).

    Tensors are float64 CUDA tensors of shape (4, nx, ny) (eta, X, X_al,
    X_th); coefficient rows are 15 float64 values. Every call runs on torch's
    current CUDA stream (kks_adj_set_stream) and returns once its work is
    queued: the results are ordered for whatever torch does next on that
    stream, and nothing waits on the host (a run of steps is launch-bound, not
    bound by a host round trip per step)."""

    def __init__(self, nx, ny, C11_0, C12_0, C44_0, device=0, surf_scale=1.0, precision="fp64"):
        self.lib = L.load()
        self.nx, self.ny, self.device = int(nx), int(ny), int(device)
        self.surf_scale = float(surf_scale)  # dx^2 / (2 lambda): interface cells -> interface measure
        h = ctypes.c_void_p()
        L.check(self.lib.kks_adj_create(self.nx, self.ny, float(C11_0), float(C12_0), float(C44_0), self.device,
                                        ctypes.byref(h)), "kks_adj_create")
        self.h = h
        self.precision = precision
        self._stream = None
        if precision != "fp64":
            code = {"mixed": L.KKS_PRECISION_MIXED}[precision]
            L.check(self.lib.kks_adj_set_precision(self.h, code), "kks_adj_set_precision")

    @classmethod
    def for_config(cls, cfg, tables, device=0, precision="fp64"):
        """Stiffness frozen at T(t = 0) (pf_kks/solver.py:152-154). ``precision``:
        "fp64" or "mixed" (FP32 transforms of the increments, FP64 elsewhere)."""
        T0 = float(np.interp(0.0, np.asarray(cfg.schedule_time, float), np.asarray(cfg.schedule_temperature, float)))
        return cls(cfg.nx, cfg.ny, tables.at(T0, "C11"), tables.at(T0, "C12"), tables.at(T0, "C44"), device,
                   surf_scale=cfg.dx**2 / (2 * cfg.lambd), precision=precision)

    def _check(self, *tensors):
        torch = _torch()
        for t in tensors:
            if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or t.numel() != 4 * self.nx * self.ny:
                raise ValueError("state tensors must be contiguous float64 CUDA tensors of 4 * nx * ny values")
        stream = torch.cuda.current_stream(self.device).cuda_stream
        if stream == 0:
            # torch's default is the legacy default stream; NULL would select
            # the handle's own (non-blocking) stream, so name the legacy one
            # (cudaStreamLegacy) to stay ordered with torch's work
            stream = 1
        if stream != self._stream:
            L.check(self.lib.kks_adj_set_stream(self.h, ctypes.c_void_p(stream)), "kks_adj_set_stream")
            self._stream = stream

    @staticmethod
    def _row(coef):
        row = np.ascontiguousarray(np.asarray(coef, dtype=np.float64).reshape(-1))
        if row.size != L.KKS_COEF_COUNT:
            raise ValueError(f"a coefficient row has {L.KKS_COEF_COUNT} values")
        return row

    def forward(self, state_in, coef, state_out):
        self._check(state_in, state_out)
        row = self._row(coef)
        L.check(self.lib.kks_adj_forward(self.h, ctypes.c_void_p(state_in.data_ptr()),
                                         row.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         ctypes.c_void_p(state_out.data_ptr())), "kks_adj_forward")
        return state_out

    def backward(self, state_in, state_out, coef, lam_out, lam_in):
        """lam_in <- cotangent of state_in; returns d<lam_out, state_out>/dcoef (15 values)."""
        self._check(state_in, state_out, lam_out, lam_in)
        row = self._row(coef)
        d = np.zeros(L.KKS_COEF_COUNT, dtype=np.float64)
        L.check(self.lib.kks_adj_backward(self.h, ctypes.c_void_p(state_in.data_ptr()),
                                          ctypes.c_void_p(state_out.data_ptr()),
                                          row.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          ctypes.c_void_p(lam_out.data_ptr()), ctypes.c_void_p(lam_in.data_ptr()),
                                          d.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "kks_adj_backward")
        return d

    def backward_into(self, state_in, state_out, coef, lam_out, lam_in, dcoef):
        """backward() with the 15 gradient values written into ``dcoef``, a
        float64 CUDA tensor of KKS_COEF_COUNT values, by the stream."""
        self._check(state_in, state_out, lam_out, lam_in)
        torch = _torch()
        if dcoef.dtype != torch.float64 or not dcoef.is_cuda or not dcoef.is_contiguous() or \
                dcoef.numel() != L.KKS_COEF_COUNT:
            raise ValueError("dcoef must be a contiguous float64 CUDA tensor of KKS_COEF_COUNT values")
        row = self._row(coef)
        L.check(self.lib.kks_adj_backward_device(self.h, ctypes.c_void_p(state_in.data_ptr()),
                                                 ctypes.c_void_p(state_out.data_ptr()),
                                                 row.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                 ctypes.c_void_p(lam_out.data_ptr()),
                                                 ctypes.c_void_p(lam_in.data_ptr()),
                                                 ctypes.c_void_p(dcoef.data_ptr())), "kks_adj_backward_device")
        return dcoef

    def close(self):
        if getattr(self, "h", None):
            self.lib.kks_adj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _histories(state):
    """eta_mean and X_al_mean of a state (pf_kks/solver.py:380-390)."""
    torch = _torch()
    eta, X = state[0], state[1]
    mask = eta < 0.05
    cnt = mask.sum()
    xal = torch.where(cnt > 0, (X * mask).sum() / cnt.clamp(min=1), torch.full((), float("nan"), dtype=X.dtype,
                                                                                device=X.device))
    return eta.mean(), xal, mask, cnt


def _interface_cells(eta):
    """Cells (nx-1)(ny-1) whose four corners lie in 0.1 <= eta <= 0.9
    (pf_kks/microstructure.py:117-128)."""
    s = (eta >= 0.1) & (eta <= 0.9)
    return (s[:-1, :-1] & s[1:, :-1] & s[1:, 1:] & s[:-1, 1:]).sum()


def _make_function():
    torch = _torch()

    class FixedDtRun(torch.autograd.Function):
        """Fixed-dt run on the GPU with the hand-written adjoint.

        forward(coef (n, 15) float64, state0 (4, nx, ny) float64 CUDA,
        stepper: StepAdjoint, checkpoint_every: int) returns eta_mean (n),
        X_al_mean (n), surf (n) (histories of the input state of each step,
        on the state's device; surf is the interface measure, a cell count
        with no gradient) and the final state (4, nx, ny)."""

        @staticmethod
        def forward(ctx, coef, state0, stepper, checkpoint_every=10):
            n = coef.shape[0]
            K = max(1, int(checkpoint_every))
            c = coef.detach().cpu().numpy()
            s = state0.detach().contiguous().clone()
            ckpt = {0: s.clone()}
            eta_mean = torch.empty(n, dtype=torch.float64, device=s.device)
            xal_mean = torch.empty(n, dtype=torch.float64, device=s.device)
            surf = torch.empty(n, dtype=torch.float64, device=s.device)
            for i in range(n):
                em, xm, _, _ = _histories(s)
                eta_mean[i] = em
                xal_mean[i] = xm
                surf[i] = _interface_cells(s[0]) * stepper.surf_scale
                nxt = torch.empty_like(s)
                stepper.forward(s, c[i], nxt)
                s = nxt
                if (i + 1) % K == 0 and i + 1 < n:
                    ckpt[i + 1] = s.clone()
            ctx.stepper = stepper
            ctx.K = K
            ctx.ckpt = ckpt
            ctx.coef_np = c
            ctx.coef_shape = coef.shape
            ctx.coef_dtype = coef.dtype
            ctx.mark_non_differentiable(surf)
            return eta_mean, xal_mean, surf, s

        @staticmethod
        def backward(ctx, g_eta, g_xal, g_surf, g_final):
            stepper, K, c = ctx.stepper, ctx.K, ctx.coef_np
            n = c.shape[0]
            s0 = ctx.ckpt[0]
            N = s0[0].numel()
            lam = torch.zeros_like(s0) if g_final is None else g_final.detach().contiguous().clone()
            grad_coef = torch.zeros(c.shape, dtype=torch.float64, device=s0.device)
            starts = sorted(ctx.ckpt)
            for seg in reversed(range(len(starts))):
                a = starts[seg]
                b = starts[seg + 1] if seg + 1 < len(starts) else n
                states = [ctx.ckpt[a]]
                for i in range(a, b):  # recompute the segment
                    nxt = torch.empty_like(states[-1])
                    stepper.forward(states[-1], c[i], nxt)
                    states.append(nxt)
                for i in reversed(range(a, b)):
                    lam_in = torch.empty_like(lam)
                    stepper.backward_into(states[i - a], states[i - a + 1], c[i], lam, lam_in, grad_coef[i])
                    # history seeds of the step's input state
                    if g_eta is not None:
                        lam_in[0] += g_eta[i] / N
                    if g_xal is not None:
                        # X_al_mean is the mean over eta < 0.05 (NaN, with no gradient, when no point is)
                        _, _, mask, cnt = _histories(states[i - a])
                        w = torch.where(cnt > 0, g_xal[i] / cnt.clamp(min=1), torch.zeros((), dtype=lam_in.dtype,
                                                                                          device=lam_in.device))
                        lam_in[1] += w * mask.to(lam_in.dtype)
                    lam = lam_in
            gc = grad_coef.to(device="cpu", dtype=ctx.coef_dtype).reshape(ctx.coef_shape)
            return gc, lam, None, None

    return FixedDtRun


_FN = None


def __getattr__(name):
    # FixedDtRun is built on first use so that importing this module does not import torch
    global _FN
    if name == "FixedDtRun":
        if _FN is None:
            _FN = _make_function()
        return _FN
    raise AttributeError(name)


def dsc_of_run(cfg, tables, state0, stepper, n_steps, theta, checkpoint_every=50, params=None,
               return_run=False):
    """Simulated DSC (:func:`pf_kks_gpu.dsc.simulated_dsc`) of a fixed-dt run
    of ``n_steps`` from ``state0`` ((4, nx, ny) float64 CUDA tensor), as a
    differentiable function of ``theta`` = (log c_D, log annealing rate,
    log c_gamma) offsets (a float64 tensor of 3). ``params``: DSCParameters
    (default: for_config(cfg)). With ``return_run`` also returns
    (eta_mean, X_al_mean, surf, final, time, T)."""
    from .dsc import DSCParameters, simulated_dsc

    coef, t, T = coefficients(cfg, tables, n_steps, log_c_D=theta[0], log_anneal=theta[1], log_c_gamma=theta[2],
                              return_times=True)
    em, xm, surf, fin = __getattr__("FixedDtRun").apply(coef, state0, stepper, checkpoint_every)
    p = DSCParameters.for_config(cfg) if params is None else params
    q = simulated_dsc(em, xm, surf, t.to(em.device), T.to(em.device), p)
    if return_run:
        return q, (em, xm, surf, fin, t, T)
    return q


def initial_state_tensor(eta, X, X_al, X_th, device=0):
    """(4, nx, ny) float64 CUDA tensor from four (nx, ny[, 1]) arrays."""
    torch = _torch()
    arrs = [np.asarray(a, dtype=np.float64).reshape(np.asarray(eta).shape[0], np.asarray(eta).shape[1])
            for a in (eta, X, X_al, X_th)]
    return torch.tensor(np.stack(arrs), dtype=torch.float64, device=f"cuda:{device}").contiguous()

