"""Calibration harness: the lattice-strain objective of a replay as a
``torch.autograd.Function``.

The device library computes the objective and its gradients in one call
(``fas_gpu_adjoint_grad``: a replay of every Gauss point's strain history,
then the reverse sweep through the converged constitutive updates).  This
wrapper lets an optimiser in torch drive the starting orientations and slip
resistances; torch is the harness here, not the compute path.
"""
from __future__ import annotations

import itertools

import numpy as np
import torch

from .solver import GpuSolver, ReplayHistory


def bunge_matrix(euler: np.ndarray) -> np.ndarray:
    """CTMATRX's a (src/fasolt/crys_math.f90:25-62) for [n, 3] Euler angles:
    [n, 3, 3]; a crystal-frame vector v has sample-frame components a^T v
    (as BTMATRX rotates the slip systems)."""
    ph1, phi, ph2 = euler[:, 0], euler[:, 1], euler[:, 2]
    c1, s1, c2, s2, c, s = np.cos(ph1), np.sin(ph1), np.cos(ph2), np.sin(ph2), np.cos(phi), np.sin(phi)
    a = np.empty((euler.shape[0], 3, 3))
    a[:, 0, 0] = c1 * c2 - s1 * s2 * c
    a[:, 1, 0] = -c1 * s2 - s1 * c2 * c
    a[:, 2, 0] = s1 * s
    a[:, 0, 1] = s1 * c2 + c1 * s2 * c
    a[:, 1, 1] = -s1 * s2 + c1 * c2 * c
    a[:, 2, 1] = -c1 * s
    a[:, 0, 2] = s2 * s
    a[:, 1, 2] = c2 * s
    a[:, 2, 2] = c
    return a


def cubic_family(hkl) -> np.ndarray:
    """The distinct plane normals of a cubic {hkl} family (unit vectors,
    one of each +/- pair)."""
    out = []
    for p in itertools.permutations(hkl):
        for sg in itertools.product((1, -1), repeat=3):
            v = np.array(p, float) * sg
            v /= np.linalg.norm(v)
            if not any(abs(abs(v @ u) - 1.0) < 1e-12 for u in out):
                out.append(v)
    return np.array(out)


def bin_weights(euler: np.ndarray, normals: np.ndarray, q, tol_deg: float) -> np.ndarray:
    """Weights of an orientation bin for the replay objective: 1/count for
    the GPs that have a plane normal of the family (crystal frame,
    `normals` [m, 3]) within tol_deg of the scattering direction q, 0 for
    the others (as a diffraction measurement selects grains)."""
    q = np.asarray(q, float) / np.linalg.norm(q)
    n = normals / np.linalg.norm(normals, axis=1, keepdims=True)
    a = bunge_matrix(np.asarray(euler, float))
    sample = np.einsum("gij,mi->gmj", a, n)             # a^T n for every GP and normal
    cosang = np.abs(sample @ q).max(axis=1)
    inside = cosang >= np.cos(np.radians(tol_deg)) - 1e-15
    w = np.zeros(len(cosang))
    if inside.any():
        w[inside] = 1.0 / inside.sum()
    return w


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
