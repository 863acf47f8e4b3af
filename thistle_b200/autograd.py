"""torch.autograd binding of the total-j0 intensity and its adjoint, on the
device.

``intensity_batch(R, plan, atom_of)`` returns I(q) of G geometries for
nuclear coordinates ``R`` (a (G, natoms, 3) float64 CUDA tensor) with every
Gaussian centre on its atom; ``intensity(R, plan, atom_of)`` is the same for
one geometry (R of shape (natoms, 3)).  The forward pass gathers the
function centres from R on the device, hands them to the plan
(``thistle_plan_set_centres_batch_device``) and runs the integrator into a
device tensor (``thistle_plan_execute_batch_device``); the backward pass runs
the library's adjoint on the incoming gradient in device memory
(``thistle_plan_vjp_batch_device``: sum_q v(q) dI/dA for every group centre)
and sums the group gradients onto their atoms with ``index_add_``.  Nothing
is copied to the host: the plan runs on the caller's current CUDA stream,
so the graph stays stream-ordered.  The pair density is held fixed.
"""
from __future__ import annotations

import numpy as np
import torch

from .main_calculation import ScatteringPlan


def _prepare(plan: ScatteringPlan, G: int, device):
    """Puts the plan on the current stream and sizes its geometry batch."""
    stream = torch.cuda.current_stream(device).cuda_stream
    if getattr(plan, "_torch_stream", None) != stream:
        plan.set_stream(stream)
        plan._torch_stream = stream
    if plan.ngeom != G:
        plan.set_batch(G)
    if not hasattr(plan, "_token"):
        plan._token = 0


def _index(a, device):
    return torch.as_tensor(np.asarray(a), dtype=torch.long, device=device)


class BatchedScatteringIntensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, R, plan: ScatteringPlan, atom_of, group_atom):
        if not R.is_cuda or R.dtype != torch.float64 or R.dim() != 3:
            raise ValueError("R must be a (G, natoms, 3) float64 CUDA tensor")
        G = R.shape[0]
        _prepare(plan, G, R.device)
        xyz = R.detach().index_select(1, atom_of).contiguous()  # (G, ngto, 3)
        plan.set_centres_batch_device(xyz.data_ptr())
        out = torch.empty((G, plan.nq), dtype=torch.float64, device=R.device)
        plan.execute_batch_device(out.data_ptr())
        plan._token += 1
        ctx.plan, ctx.token, ctx.natoms = plan, plan._token, R.shape[1]
        ctx.save_for_backward(xyz, group_atom)
        return out

    @staticmethod
    def backward(ctx, gI):
        plan = ctx.plan
        xyz, group_atom = ctx.saved_tensors
        G = xyz.shape[0]
        _prepare(plan, G, gI.device)
        if plan._token != ctx.token:
            # another forward moved the plan since: restore this one's centres
            plan.set_centres_batch_device(xyz.data_ptr())
            plan._token += 1
            ctx.token = plan._token
        v = gI.detach().to(torch.float64).contiguous()
        gg = torch.empty((G, plan.ng, 3), dtype=torch.float64, device=gI.device)
        plan.vjp_batch_device(v.data_ptr(), gg.data_ptr())
        gR = torch.zeros((G, ctx.natoms, 3), dtype=torch.float64, device=gI.device)
        gR.index_add_(1, group_atom, gg)
        return gR, None, None, None


def intensity_batch(R: torch.Tensor, plan: ScatteringPlan, atom_of) -> torch.Tensor:
    """I(q) of the plan's basis and density at nuclear coordinates R
    ((G, natoms, 3), CUDA, float64), shape (G, nq); differentiable in R."""
    atom_of = np.asarray(atom_of)
    a = _index(atom_of, R.device)
    ga = _index(atom_of[plan.group_first], R.device)
    return BatchedScatteringIntensity.apply(R, plan, a, ga)


def intensity(R: torch.Tensor, plan: ScatteringPlan, atom_of) -> torch.Tensor:
    """I(q) at nuclear coordinates R ((natoms, 3), CUDA, float64); differentiable in R."""
    return intensity_batch(R.unsqueeze(0), plan, atom_of)[0]
