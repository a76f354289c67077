"""The energy as a differentiable torch function of the coordinates.

``energy(xyz, batch)`` returns the per-system total energies of the
coordinates ``xyz`` ([natoms, 3], float64, CUDA) — calculate_potential
semantics: a fresh neighbor list, HCT Born radii, pair sum, SASA,
dihedrals, disulfides (physics_engine.cpp:2205-2248).  Its backward is the
hand-written gradient kernel (alma_forces), scaled per system by the
incoming gradient; the gradient is computed in the forward pass (the batch
holds one geometry at a time, so the backward must not depend on it).

    from protein_physics_b200.autograd import EnergyModel
    model = EnergyModel([(xyz, q, r, eps, flat)], precision="fp64")
    x = model.coords().requires_grad_()
    E = model(x).sum()
    E.backward()          # x.grad = dE/dx
"""
from __future__ import annotations

import torch

from .device import DeviceBatch


class _Energy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyz, batch, graph):
        n = batch.natoms
        if xyz.shape != (n, 3) or xyz.dtype != torch.float64 or not xyz.is_cuda:
            raise ValueError(f"xyz must be a CUDA float64 tensor of shape ({n}, 3)")
        batch.xyz[:n, :3].copy_(xyz.detach())
        if graph:  # list, radii, energy and gradient as one replayed CUDA graph
            terms, grad = batch.evaluate(graph=True)
            if ctx.needs_input_grad[0]:
                ctx.save_for_backward(grad[:n, :3].clone(), batch.atom_sys)
            return terms[:, 4].clone()
        batch.nl_ready = False
        batch.invalidate_sasa()
        batch.build_nl()
        terms = batch.energy_terms(recompute_born=True)
        if ctx.needs_input_grad[0]:
            g = batch.forces()[:n, :3].clone()
            ctx.save_for_backward(g, batch.atom_sys)
        return terms[:, 4].clone()

    @staticmethod
    def backward(ctx, gE):
        g, sys_of = ctx.saved_tensors
        return g * gE[sys_of].unsqueeze(1), None, None


def energy(xyz, batch: DeviceBatch, graph=False):
    """Per-system total energies [nsys] of coordinates xyz [natoms, 3]
    (graph=True: evaluated by replaying one captured CUDA graph)."""
    return _Energy.apply(xyz, batch, bool(graph))


class EnergyModel(torch.nn.Module):
    """A fixed set of systems (parameters and topology) whose energy is a
    differentiable function of the coordinates."""

    def __init__(self, systems, precision="mixed", graph=False):
        super().__init__()
        self.batch = DeviceBatch(systems, precision=precision)
        self.graph = bool(graph)

    def coords(self):
        return self.batch.xyz[:self.batch.natoms, :3].clone()

    def forward(self, xyz):
        return energy(xyz, self.batch, self.graph)
