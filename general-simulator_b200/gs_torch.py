"""torch.autograd bridge to the hand-written adjoint of the martensite run.

Used by calibration and tests only: the forward and backward sweeps are the
C ABI's gs_adjoint_forward / gs_adjoint_backward (CUDA), and torch only
carries the tensors and composes the loss.  The parameter vector is

    theta = (kappa, A2, A4, A6, Ac, m)

with m the eigenstrain magnitude: every variant's eigenstrain is m times a
fixed shape (the eigenstrains given at construction divided by m0, the
largest absolute entry among them).
"""
from __future__ import annotations

import numpy as np
import torch

import gs_b200 as gb


class MartensiteRun:
    """A fixed grid, step count and checkpoint interval; theta varies."""

    def __init__(self, params: gb.GsParams, nsteps: int, checkpoint_every: int):
        self.base = params.copy()
        eps = self.base.get_eigenstrain()
        self.m0 = float(np.abs(eps).max())
        self.shape_eps = eps / self.m0
        self.adj = gb.Adjoint(self.base, nsteps, checkpoint_every)
        self.m = self.m0

    def theta0(self) -> torch.Tensor:
        p = self.base
        return torch.tensor([p.kappa, p.landau[0], p.landau[1], p.landau[2], p.landau[3], self.m0],
                            dtype=torch.float64)

    def params_for(self, theta) -> gb.GsParams:
        t = [float(x) for x in theta]
        p = self.base.copy()
        p.kappa = t[0]
        for i in range(4):
            p.landau[i] = t[1 + i]
        p.set_eigenstrain(self.shape_eps * t[5])
        return p

    def close(self) -> None:
        self.adj.close()


class _Run(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eta0: torch.Tensor, theta: torch.Tensor, run: MartensiteRun):
        run.adj.set_params(run.params_for(theta.detach()))
        run.m = float(theta[5])
        eT, eel = run.adj.forward(eta0.detach().to(torch.float64).cpu().numpy())
        ctx.run = run
        ctx.eta_dtype = eta0.dtype
        return torch.from_numpy(eT).to(eta0.dtype), torch.tensor(eel, dtype=torch.float64)

    @staticmethod
    def backward(ctx, g_eta, g_e):
        run = ctx.run
        if g_eta is None:
            seed = np.zeros(run.adj.shape)
        else:
            seed = g_eta.detach().to(torch.float64).cpu().numpy()
        se = 0.0 if g_e is None else float(g_e)
        _, g, ge = run.adj.backward(seed=seed, seed_e=se)
        gt = g.copy()
        gt[5] = g[5] / run.m  # d/dm = (d/ds) / m at s = 1
        return torch.from_numpy(ge).to(ctx.eta_dtype), torch.from_numpy(gt), None


def martensite_run(eta0: torch.Tensor, theta: torch.Tensor, run: MartensiteRun):
    """(eta_T, E_el(T)) of the run from eta0 with parameters theta; both
    differentiable with respect to eta0 and theta."""
    return _Run.apply(eta0, theta, run)


def calibration_loss(eta_T, e_el, target, e_target, lam_el):
    """||eta_T - target||^2 + lam_el (E_el(T) - E_target)^2."""
    return ((eta_T - target) ** 2).sum() + lam_el * (e_el - e_target) ** 2


def calibration_setup(n: int = 96, nsteps: int = 200, dtype: int = gb.GS_DTYPE_F32, checkpoint_every: int = 20):
    """The calibration workload: 3-variant martensite on an n^3 grid, nsteps
    steps of dt = 0.005, noise off.  The target (eta_T and E_el(T)) is a
    forward run at perturbed parameters (kappa 0.8, A2 0.25, eigenstrain
    magnitude 0.022) from eta ~ U[-0.01, 0.01] with seed 3; the run to
    calibrate starts from U[-0.01, 0.01] with seed 4.  Returns (run, theta0,
    eta0, target, e_target)."""
    p = gb.mart3d_params(n, dtype=dtype, noise=0.0)
    run = MartensiteRun(p, nsteps, checkpoint_every)
    th_t = run.theta0().clone()
    th_t[0], th_t[1], th_t[5] = 0.8, 0.25, 0.022
    run.adj.set_params(run.params_for(th_t))
    target, e_target = run.adj.forward(gb.initial_eta(p, 3, 0.01))
    eta0 = gb.initial_eta(p, 4, 0.01)
    return run, run.theta0(), eta0, target, e_target
