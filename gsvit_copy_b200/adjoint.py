"""Thin torch.autograd wrapper of the library's discrete adjoint
(fdtd_adjoint_gradient): J(eps_r) of a design region with its gradient.

No counterpart in the reference.  The forward call restores the solver's
initial state, sets the design permittivities and runs the checkpointed
forward + adjoint sweep on the GPU; backward returns dJ/d eps_r scaled by the
incoming gradient.  Meant for checking the adjoint (finite differences, the
FP64 CPU adjoint), not for training loops."""
from __future__ import annotations

import numpy as np


def objective_function():
    import torch

    class FarFieldObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, eps, solver, obj, nsteps, checkpoint, initial_state):
            solver.restore(initial_state)
            solver.set_design_eps(eps.detach().cpu().numpy().astype(np.float64))
            J, grad = solver.adjoint_gradient(obj, nsteps, checkpoint)
            ctx.save_for_backward(torch.from_numpy(grad).to(eps.device, eps.dtype))
            return eps.new_tensor(J)

        @staticmethod
        def backward(ctx, gJ):
            (grad,) = ctx.saved_tensors
            return gJ * grad, None, None, None, None, None

    return FarFieldObjective


def far_field_objective(eps, solver, obj: dict, nsteps: int, checkpoint: int = 200, initial_state=None):
    """J(eps) as a differentiable torch scalar; `initial_state` is a snapshot of
    the solver to start every evaluation from (taken now when omitted)."""
    if initial_state is None:
        initial_state = solver.snapshot()
    return objective_function().apply(eps, solver, obj, nsteps, checkpoint, initial_state)
