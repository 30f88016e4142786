"""Calibration harness: the lattice-strain objective of a replay as a
``torch.autograd.Function``.

The device library computes the objective and its gradients in one call
(``fas_gpu_adjoint_grad``: a replay of every Gauss point's strain history,
then the reverse sweep through the converged constitutive updates).  This
wrapper lets an optimiser in torch drive the starting orientations and slip
resistances; torch is the harness here, not the compute path.
"""
from __future__ import annotations

import torch

from .solver import GpuSolver, ReplayHistory


class LatticeStrainObjective(torch.autograd.Function):
    """J(euler, crss) for a solver and a replay history.

    euler [ngps, 3] and crss [ngps, ns] (float64, CPU) replace the starting
    Euler angles and slip resistances in the solver's state (sv(1:3) and
    sv(4:3+ns)); the rest of the state (stress, other variables) stays as
    the solver's problem holds it.  backward returns dJ/deuler and dJ/dcrss
    from the adjoint."""

    @staticmethod
    def forward(ctx, euler: torch.Tensor, crss: torch.Tensor, solver: GpuSolver,
                hist: ReplayHistory) -> torch.Tensor:
        p = solver.prob
        ns = crss.shape[1]
        p.sv[:, 0:3] = euler.detach().cpu().double().numpy()
        p.sv[:, 3:3 + ns] = crss.detach().cpu().double().numpy()
        solver.upload(p)
        out = solver.adjoint_grad(hist)
        ctx.save_for_backward(torch.from_numpy(out["sv"][:, 0:3].copy()),
                              torch.from_numpy(out["sv"][:, 3:3 + ns].copy()))
        return torch.tensor(out["J"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_j: torch.Tensor):
        g_euler, g_crss = ctx.saved_tensors
        return grad_j * g_euler, grad_j * g_crss, None, None
