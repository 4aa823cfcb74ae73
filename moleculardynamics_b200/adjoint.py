"""Fitting helpers on top of the differentiable LJ trajectory (no reference
counterpart).

`LJTrajectory` is a torch.autograd.Function: its forward runs the FP64
velocity-Verlet trajectory on the GPU through md_adjoint_forward (saving states
every `every` steps for backward) and returns the per-step rows [U, W, KE]; its
backward calls md_adjoint_backward, which recomputes each segment from its saved
state and walks the hand-written adjoint back through it.  PyTorch is only the
autograd plumbing here: tensors cross to the library as host arrays.

`pressure_energy_loss` is the loss the fitting workload uses: the squared
mismatch of the time-averaged virial pressure and potential energy per atom
against targets, with the analytic long-range corrections of a truncated
potential (forcefield/lennard_jones.cpp:121-151) written as differentiable
expressions in epsilon and sigma.
"""
import math

import numpy as np

import moleculardynamics_b200 as md


def tail_corrections(eps, sigma, rc, n, volume, truncation):
    """U_LRC and P_LRC (lennard_jones.cpp:121-151); zero for the force-shifted
    potential.  Works on floats and on torch tensors."""
    if truncation == md.Truncation.LinearForceShift:
        return 0.0 * eps, 0.0 * eps
    rho = n / volume
    sr = sigma / rc
    sr3 = sr * sr * sr
    sr9 = sr3 * sr3 * sr3
    sig3 = sigma * sigma * sigma
    u = (8.0 / 3.0) * math.pi * n * rho * eps * sig3 * ((1.0 / 3.0) * sr9 - sr3)
    p = (16.0 / 3.0) * math.pi * rho * rho * eps * sig3 * ((2.0 / 3.0) * sr9 - sr3)
    return u, p


def pressure_energy_loss(rows, eps, sigma, rc, n, volume, dof, truncation, p_target, u_target,
                         w_p=1.0, w_u=1.0):
    """L = w_p (mean_k P_k - p_target)^2 + w_u (mean_k u_k - u_target)^2 with
    P_k = rho T_k + W_k / (3V) + P_LRC, T_k = 2 KE_k / dof, u_k = (U_k + U_LRC) / n
    (apps/moldyn_run.cpp:497-511).  Works on numpy arrays and torch tensors."""
    u_lrc, p_lrc = tail_corrections(eps, sigma, rc, n, volume, truncation)
    rho = n / volume
    p_k = rho * (2.0 * rows[:, 2] / dof) + rows[:, 1] / (3.0 * volume) + p_lrc
    u_k = (rows[:, 0] + u_lrc) / n
    return w_p * (p_k.mean() - p_target) ** 2 + w_u * (u_k.mean() - u_target) ** 2


def loss_and_gradients(sys, lj_params, dt, steps, every, skin, p_target, u_target, ctx=None,
                       w_p=1.0, w_u=1.0):
    """Runs the trajectory from `sys` and returns (loss, dL/d epsilon, dL/d sigma,
    dL/dx0 (N, 3), rows) with numpy only: the adjoint of the per-step rows plus the
    analytic tail-correction terms.  lj_params = (epsilon, sigma, rc, truncation).
    The system is left at the end of the trajectory."""
    eps, sigma, rc, trunc = lj_params
    lj = md.LennardJones(sigma, eps, rc, trunc)
    traj = md.AdjointTrajectory(ctx or sys.ctx)
    rows = traj.forward(sys, lj, dt, steps, every, skin)
    n, vol = sys.n, sys.volume()
    dof = 3 * n - 3
    u_lrc, p_lrc = tail_corrections(eps, sigma, rc, n, vol, trunc)
    rho = n / vol
    p_mean = (rho * 2.0 * rows[:, 2] / dof + rows[:, 1] / (3.0 * vol)).mean() + p_lrc
    u_mean = ((rows[:, 0] + u_lrc) / n).mean()
    loss = w_p * (p_mean - p_target) ** 2 + w_u * (u_mean - u_target) ** 2
    dp = 2.0 * w_p * (p_mean - p_target)
    du = 2.0 * w_u * (u_mean - u_target)
    g = np.zeros_like(rows)
    g[:, 0] = du / (n * steps)
    g[:, 1] = dp / (3.0 * vol * steps)
    g[:, 2] = dp * rho * 2.0 / (dof * steps)
    d_eps, d_sig, gx, _ = traj.backward(g)
    if trunc != md.Truncation.LinearForceShift:
        # tail terms: linear in epsilon; d/d sigma from the closed forms
        d_eps += dp * p_lrc / eps + du * u_lrc / (n * eps)
        sr3, sr9 = (sigma / rc) ** 3, (sigma / rc) ** 9
        du_lrc = (8.0 / 3.0) * math.pi * n * rho * eps * (4.0 * sr9 * sigma ** 2 - 6.0 * sr3 * sigma ** 2)
        dp_lrc = (16.0 / 3.0) * math.pi * rho * rho * eps * (8.0 * sr9 * sigma ** 2 - 6.0 * sr3 * sigma ** 2)
        d_sig += dp * dp_lrc + du * du_lrc / n
    return loss, d_eps, d_sig, gx, rows


def _torch_function():
    import torch

    class LJTrajectory(torch.autograd.Function):
        """rows = LJTrajectory.apply(eps, sigma, x0, v0, cfg): (steps, 3) tensor of
        [U, W, KE]; differentiable in eps, sigma, x0 and v0 (cfg: dict with keys
        masses, box, rc, truncation, dt, steps, every, skin, context)."""

        @staticmethod
        def forward(ctx, eps, sigma, x0, v0, cfg):
            sys = md.System.from_arrays(x0.detach().cpu().numpy(), cfg["box"],
                                        vel=v0.detach().cpu().numpy(), mass=cfg["masses"],
                                        ctx=cfg.get("context"))
            lj = md.LennardJones(float(sigma), float(eps), cfg["rc"], cfg["truncation"])
            traj = md.AdjointTrajectory(sys.ctx)
            rows = traj.forward(sys, lj, cfg["dt"], cfg["steps"], cfg.get("every", 50),
                                cfg.get("skin", 1.0))
            ctx.traj = traj
            ctx.keep = (sys, lj)  # save-for-backward: the trajectory's saved states
            return torch.as_tensor(rows, dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_rows):
            d_eps, d_sig, gx, gv = ctx.traj.backward(grad_rows.detach().cpu().numpy())
            return (torch.tensor(d_eps, dtype=torch.float64),
                    torch.tensor(d_sig, dtype=torch.float64),
                    torch.as_tensor(gx), torch.as_tensor(gv), None)

    return LJTrajectory


_LJTrajectory = None


def __getattr__(name):
    global _LJTrajectory
    if name == "LJTrajectory":
        if _LJTrajectory is None:
            _LJTrajectory = _torch_function()
        return _LJTrajectory
    raise AttributeError(name)
