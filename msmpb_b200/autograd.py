"""torch.autograd binding: energy and forces of the MSM evaluation as a
differentiable function of positions and charges.

``msm_energy_forces(ff, positions, charges)`` returns ``(U, F)`` (a 0-d
tensor and an (N, 3) tensor, FP64, on the GPU of ``ff``). Backward maps the
cotangents (Ubar, Fbar) to

  dL/dq = Ubar phi + (charge part of the adjoint),
  dL/dr = -Ubar F + (position part of the adjoint),

where the adjoint part (the transposed operator chain, hand-written CUDA)
comes from ``FF_adjoint_device`` with Ubar = 0 and the Ubar terms are added
here from the forward's potentials and forces (no host synchronisation).
The adjoint reuses the forward's grids when no other evaluation ran on the
handle in between (``FF_evaluation_count``), else it reruns the forward.
"""
import torch

from .forcefield import ForceField


class MSMEnergyForces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, charges, ff, weights=None):
        pos = positions.detach().contiguous().to(torch.float64)
        q = charges.detach().contiguous().to(torch.float64)
        n = pos.shape[0]
        f = torch.empty((n, 3), dtype=torch.float64, device=pos.device)
        phi = torch.empty(n, dtype=torch.float64, device=pos.device)
        e = torch.empty(1, dtype=torch.float64, device=pos.device)
        stream = torch.cuda.current_stream(pos.device).cuda_stream
        ff.energy_device(pos.data_ptr(), q.data_ptr(), f.data_ptr(), phi.data_ptr(),
                         e.data_ptr(), stream, weights=weights)
        ctx.ff = ff
        ctx.weights = weights
        ctx.count = ff.evaluation_count()
        ctx.save_for_backward(pos, q, f, phi)
        return e[0], f

    @staticmethod
    def backward(ctx, g_energy, g_force):
        pos, q, f, phi = ctx.saved_tensors
        ff = ctx.ff
        if g_force is None:
            g_force = torch.zeros_like(f)
        fbar = g_force.contiguous().to(torch.float64)
        dq = torch.empty_like(q)
        dr = torch.empty_like(pos)
        stream = torch.cuda.current_stream(pos.device).cuda_stream
        reuse = ff.evaluation_count() == ctx.count
        ff.adjoint_device(pos.data_ptr(), q.data_ptr(), fbar.data_ptr(), 0.0, dq.data_ptr(),
                          dr.data_ptr(), reuse=reuse, stream=stream, weights=ctx.weights)
        if g_energy is not None:
            dq = dq + g_energy * phi
            dr = dr - g_energy * f
        return dr, dq, None, None


def msm_energy_forces(ff: ForceField, positions, charges, weights=None):
    """(U, F) with autograd support for positions and charges."""
    return MSMEnergyForces.apply(positions, charges, ff, weights)
