"""torch.autograd binding of the total-j0 intensity and its adjoint.

``ScatteringIntensity.apply(R, plan, atom_of)`` returns I(q) for nuclear
coordinates ``R`` (natoms x 3, float64) with every Gaussian centre on its
atom; its backward pass calls the library's adjoint
(``thistle_plan_vjp``: sum_q v(q) dI/dA for each group centre) and sums the
group gradients onto the atoms.  The pair density is held fixed.
"""
from __future__ import annotations

import numpy as np
import torch

from .main_calculation import ScatteringPlan


class ScatteringIntensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, R, plan: ScatteringPlan, atom_of):
        Rn = R.detach().cpu().numpy().astype(np.float64)
        xyz = Rn[atom_of]
        plan.set_centres(xyz[:, 0], xyz[:, 1], xyz[:, 2])
        out = plan.execute()
        ctx.plan = plan
        ctx.atom_of = atom_of
        ctx.xyz = xyz
        ctx.natoms = R.shape[0]
        return torch.as_tensor(out, dtype=R.dtype, device=R.device)

    @staticmethod
    def backward(ctx, gI):
        plan = ctx.plan
        # the plan may have been moved by another forward since: restore this one's centres
        plan.set_centres(ctx.xyz[:, 0], ctx.xyz[:, 1], ctx.xyz[:, 2])
        gg = plan.vjp(gI.detach().cpu().numpy().astype(np.float64))
        # group g's centre is that of its first function
        first = plan.group_first
        gR = np.zeros((ctx.natoms, 3))
        np.add.at(gR, ctx.atom_of[first], gg)
        return torch.as_tensor(gR, dtype=gI.dtype, device=gI.device), None, None


def intensity(R: torch.Tensor, plan: ScatteringPlan, atom_of) -> torch.Tensor:
    """I(q) of the plan's basis and density at nuclear coordinates R (differentiable in R)."""
    return ScatteringIntensity.apply(R, plan, np.asarray(atom_of))
