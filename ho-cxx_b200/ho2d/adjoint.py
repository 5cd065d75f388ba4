"""The discrete adjoint as a ``torch.autograd.Function``.

``rollout(solver, omega0, parl_vel, nsteps, ckpt_every)`` runs ``nsteps`` time steps of a
set-up :class:`ho2d.HO_2D` from the initial vorticity ``omega0`` ([N_el][K][K]) with the
wall velocity ``parl_vel`` (BC_parl_vel, [N_eb][K]) and returns omega(T). Its backward is
the library's discrete adjoint (``ho2d_adjoint_backward``): the transposed stage kernels
and one transposed Poisson solve per stage, with the forward trajectory recomputed from
checkpoints kept every ``ckpt_every`` steps. The tensors live on the host (FP64); the
solve runs on the solver's GPU.

    w0 = torch.tensor(omega0, requires_grad=True)
    pv = torch.tensor(parl_vel, requires_grad=True)
    wT = rollout(solver, w0, pv, 500, 25)
    J = 0.5 * ((wT - target) ** 2).sum()
    J.backward()            # w0.grad, pv.grad

One rollout is in flight per solver: a second forward on the same solver replaces the
checkpoints the first one's backward needs.
"""

from __future__ import annotations

import numpy as np
import torch

from . import capi


class Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, omega0, parl_vel, solver, nsteps: int, ckpt_every: int):
        solver.set_boundary(capi.BC_PARL_VEL, parl_vel.detach().cpu().double().numpy())
        solver.setsolnvort_d(omega0.detach().cpu().double().numpy())
        solver.adjoint_forward(int(nsteps), int(ckpt_every))
        ctx.solver = solver
        ctx.rollout_id = getattr(solver, "_rollouts", 0) + 1
        solver._rollouts = ctx.rollout_id
        return torch.from_numpy(np.array(solver.getallvorts_d(), copy=True))

    @staticmethod
    def backward(ctx, grad_wT):
        solver = ctx.solver
        if getattr(solver, "_rollouts", 0) != ctx.rollout_id:
            raise RuntimeError("another rollout on this solver replaced the checkpoints of this one")
        gw, gpv = solver.adjoint_backward(grad_wT.detach().cpu().double().numpy())
        return torch.from_numpy(gw), torch.from_numpy(gpv), None, None, None


def rollout(solver, omega0: torch.Tensor, parl_vel: torch.Tensor, nsteps: int, ckpt_every: int = 25) -> torch.Tensor:
    return Rollout.apply(omega0, parl_vel, solver, nsteps, ckpt_every)
