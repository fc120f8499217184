"""A torch.autograd.Function over the adjoint gradient of the slab solve,
for checking the adjoint with torch's tools (central differences,
torch.autograd.gradcheck); the gradient itself is computed by the library
(stmg_solver_gradient: one forward sweep over the slabs with checkpoints,
then the transposed space-time system solved backward over the slabs
through the same multigrid, operators.h:124-152).

J(theta) = 1/2 sum_s |U_s(theta) - O_s|^2 with theta = log(kappa) per fine
cell, U_s the slab solutions from the solver's initial state and O_s the
observations.
"""
import numpy as np
import torch


class SpaceTimeMisfit(torch.autograd.Function):
    """forward(theta, make_solver, obs, checkpoint_every) -> J.

    make_solver(kappa) returns a stmg.Solver with per-cell coefficient
    kappa = exp(theta) in its initial state; obs is (n_slabs, n_blocks *
    n_nodes). The gradient is computed with J in forward and returned by
    backward scaled by the incoming gradient."""

    @staticmethod
    def forward(ctx, theta, make_solver, obs, checkpoint_every=0):
        th = theta.detach().to("cpu", torch.float64).numpy()
        solver = make_solver(np.exp(th))
        J, grad, _, _ = solver.gradient(obs, checkpoint_every=checkpoint_every)
        ctx.save_for_backward(torch.from_numpy(grad).to(device=theta.device, dtype=theta.dtype))
        return theta.new_tensor(J)

    @staticmethod
    def backward(ctx, grad_J):
        (grad,) = ctx.saved_tensors
        return grad_J * grad, None, None, None


def misfit(theta, make_solver, obs, checkpoint_every=0):
    """J(theta) as a differentiable torch scalar (see SpaceTimeMisfit)."""
    return SpaceTimeMisfit.apply(theta, make_solver, obs, checkpoint_every)


def misfit_value(theta, make_solver, obs):
    """J(theta) by a forward solve only (no adjoint), for finite differences."""
    th = theta.detach().to("cpu", torch.float64).numpy() if torch.is_tensor(theta) else np.asarray(theta)
    solver = make_solver(np.exp(th))
    n_slabs = obs.shape[0]
    J = 0.0
    for s in range(n_slabs):
        solver.run(1)
        u, _ = solver.solution(want_v=False)
        J += 0.5 * float(np.sum((u - obs[s]) ** 2))
    return J
