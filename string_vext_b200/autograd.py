"""``PoseEnergy``: torch.autograd.Function over the hand-written adjoint.

Forward evaluates the pose energy and, in the same launch, the analytic
gradient (pair terms recomputed in the kernel, nothing stored per pair);
backward scales the saved gradients by the incoming grad.  Inputs are CUDA
float64 tensors: ``centers`` (n, 3) Cartesian A and ``quats`` (n, 4)
(w, x, y, z); the quaternion gradient is the tangent-space gradient of
E(q / |q|).  There is no CPU path: CPU tensors raise.
"""
from __future__ import annotations

import torch

from . import _lib


class PoseEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, centers, quats, system, mode=_lib.VEXT_MODE_MIXED):
        if not (centers.is_cuda and quats.is_cuda):
            raise RuntimeError("PoseEnergy runs on CUDA tensors only")
        centers = centers.detach().to(torch.float64).contiguous()
        quats = quats.detach().to(torch.float64).contiguous()
        n = centers.shape[0]
        energy = torch.empty(n, dtype=torch.float64, device=centers.device)
        gc = torch.empty((n, 3), dtype=torch.float64, device=centers.device)
        gq = torch.empty((n, 4), dtype=torch.float64, device=centers.device)
        system.pose_energy_grad_device(centers, quats, energy, gc, gq, None, mode=mode,
                                       stream=torch.cuda.current_stream(centers.device))
        ctx.save_for_backward(gc, gq)
        return energy

    @staticmethod
    def backward(ctx, grad_energy):
        gc, gq = ctx.saved_tensors
        g = grad_energy.to(torch.float64)[:, None]
        return g * gc, g * gq, None, None


def pose_energy(system, centers, quats, mode=_lib.VEXT_MODE_MIXED):
    """E(centers, quats) with autograd support."""
    return PoseEnergy.apply(centers, quats, system, mode)
