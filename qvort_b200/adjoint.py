"""Differentiable filament dynamics on top of the C ABI's hand-written derivatives.

The velocity u = calc_velocity(x) (src/timestep.f90:180-309), the energy
E = energy_info(x, u) (src/diagnostic.f90:259-280) and the position update of
pmotion with the periodic wrap (src/timestep.f90:48-71, src/periodic.f90:
188-214) are torch.autograd.Functions whose forward and backward passes are
CUDA kernels of the C ABI (qv_velocity_device / qv_velocity_vjp,
qv_energy_grad, qv_ab_step_device / qv_ab_vjp_device); torch only chains
them.  torch.utils.checkpoint keeps one state every `checkpoint_every` steps
and recomputes the steps in between during the backward pass.

With velocity Tree the topology of each step's octree is frozen in its
derivative (the opening decisions are piecewise constant in x).
"""
from __future__ import annotations

import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from . import lib as L


class FilamentSystem:
    """A fixed set of links (infront/behind) and run parameters on one GPU."""

    def __init__(self, params: L.QvParams, infront, behind, device="cuda"):
        self.params = params
        self.device = torch.device(device)
        self.inf = torch.as_tensor(np.asarray(infront, np.int32), device=self.device)
        self.beh = torch.as_tensor(np.asarray(behind, np.int32), device=self.device)
        self.n = int(self.inf.shape[0])
        self.stream = torch.cuda.current_stream(self.device)
        # The context reads and writes torch-owned device memory, so it must
        # run on torch's stream.  torch's default stream has handle 0, which
        # qv_create takes as "make a private stream": pass cudaStreamLegacy
        # (0x1), the same legacy default stream, instead.
        self.ctx = L.Context(params, stream=self.stream.cuda_stream or 0x1)

    def load(self, x: torch.Tensor):
        assert x.dtype == torch.float64 and x.is_cuda and x.shape == (self.n, 3)
        x = x.contiguous()
        self.ctx.set_points_device(self.n, x.data_ptr(), self.inf.data_ptr(), self.beh.data_ptr())
        return x

    def close(self):
        self.ctx.close()


class VelocityFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, system: FilamentSystem):
        x = system.load(x.detach())
        u = torch.empty_like(x)
        system.ctx.velocity_device(u.data_ptr())
        ctx.save_for_backward(x)
        ctx.system = system
        return u

    @staticmethod
    def backward(ctx, ubar):
        (x,) = ctx.saved_tensors
        system = ctx.system
        system.load(x)
        xbar = torch.empty_like(x)
        system.ctx.velocity_vjp(ubar.contiguous().data_ptr(), xbar.data_ptr())
        return xbar, None


class EnergyFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, u, system: FilamentSystem):
        x = system.load(x.detach())
        u = u.detach().contiguous()
        xbar = torch.empty_like(x)
        ubar = torch.empty_like(u)
        e = system.ctx.energy_grad(u.data_ptr(), xbar.data_ptr(), ubar.data_ptr())
        ctx.save_for_backward(xbar, ubar)
        return torch.tensor(e, dtype=torch.float64, device=x.device)

    @staticmethod
    def backward(ctx, ebar):
        xbar, ubar = ctx.saved_tensors
        return ebar * xbar, ebar * ubar, None


def velocity(x: torch.Tensor, system: FilamentSystem) -> torch.Tensor:
    return VelocityFn.apply(x, system)


def energy(x: torch.Tensor, u: torch.Tensor, system: FilamentSystem) -> torch.Tensor:
    return EnergyFn.apply(x, u, system)


class ABStepFn(torch.autograd.Function):
    """pmotion's position update (src/timestep.f90:48-71) and enforce_periodic
    (src/periodic.f90:188-214) as one CUDA kernel each way: the forward takes
    the update kernel's operations (bitwise the positions qv_step stores), the
    backward is the hand-written adjoint qv_ab_vjp_device."""

    @staticmethod
    def forward(ctx, x, u, u1, u2, u3, system: FilamentSystem):
        x, u, u1, u2, u3 = (t.detach().contiguous() for t in (x, u, u1, u2, u3))
        xo = torch.empty_like(x)
        system.ctx.ab_step_device(x.data_ptr(), u.data_ptr(), u1.data_ptr(), u2.data_ptr(),
                                  u3.data_ptr(), xo.data_ptr())
        ctx.save_for_backward(u1, u2, u3)
        ctx.system = system
        return xo

    @staticmethod
    def backward(ctx, xob):
        u1, u2, u3 = ctx.saved_tensors
        xob = xob.contiguous()
        out = [torch.empty_like(xob) for _ in range(5)]
        ctx.system.ctx.ab_vjp_device(u1.data_ptr(), u2.data_ptr(), u3.data_ptr(), xob.data_ptr(),
                                     *[t.data_ptr() for t in out])
        return (*out, None)


def ab_step(x, u, u1, u2, u3, system: FilamentSystem):
    """One Adams-Bashforth rung per point (exact-zero history tests) and the
    periodic wrap."""
    return ABStepFn.apply(x, u, u1, u2, u3, system)


def run(x0: torch.Tensor, system: FilamentSystem, nsteps: int, checkpoint_every: int = 16):
    """x_K after nsteps Adams-Bashforth steps from x0 with zero history."""
    zero = torch.zeros_like(x0)

    def segment(x, u1, u2, u3, k):
        for _ in range(k):
            u = velocity(x, system)
            x = ab_step(x, u, u1, u2, u3, system)
            u1, u2, u3 = u, u1, u2
        return x, u1, u2, u3

    x, u1, u2, u3 = x0, zero, zero, zero
    for s in range(0, nsteps, checkpoint_every):
        k = min(checkpoint_every, nsteps - s)
        if checkpoint_every and torch.is_grad_enabled():
            x, u1, u2, u3 = checkpoint(segment, x, u1, u2, u3, k, use_reentrant=False)
        else:
            x, u1, u2, u3 = segment(x, u1, u2, u3, k)
    return x


def min_image(d: torch.Tensor, system: FilamentSystem):
    if system.params.boundary != 1:
        return d
    L_ = system.params.box_size
    return d - L_ * torch.round(d.detach() / L_)


def loss(x0: torch.Tensor, system: FilamentSystem, nsteps: int, checkpoint_every: int = 16):
    """Filament kinetic energy (energy_info) of the final state plus the squared
    displacement of the points: E(x_K) + sum |x_K - x_0|^2."""
    xk = run(x0, system, nsteps, checkpoint_every)
    uk = velocity(xk, system)
    return energy(xk, uk, system) + (min_image(xk - x0, system) ** 2).sum()


def gradient(x0: np.ndarray, system: FilamentSystem, nsteps: int, checkpoint_every: int = 16):
    """(loss, dloss/dx0) for initial positions x0 (n, 3)."""
    x = torch.tensor(np.asarray(x0, np.float64), device=system.device, requires_grad=True)
    val = loss(x, system, nsteps, checkpoint_every)
    (g,) = torch.autograd.grad(val, x)
    return float(val.item()), g.detach().cpu().numpy()
