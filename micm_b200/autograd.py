"""torch.autograd.Function over the solver's C ABI (micmb_solve + micmb_solve_adjoint).

    y_final = RosenbrockSolve.apply(y0, log_rate_scale, solver, state, dt)

y0 is [n_cells, n_species] in the mechanism's species order, log_rate_scale
is [n_reactions] (input order); the rate constants of every cell are scaled
by exp(log_rate_scale).  The forward pass is the fused per-cell solve; the
backward pass reruns it with checkpoints and sweeps the discrete adjoint of
the accepted steps, returning dL/dy0 and dL/dlog_rate_scale (summed over
cells).  Tensors may live on the CPU or a CUDA device; the solver moves them
through host memory, as micm's own state does.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import Solver, State


class RosenbrockSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y0: torch.Tensor, log_rate_scale: torch.Tensor, solver: Solver, state: State, dt: float,
                max_checkpoints: int = 256):
        ctx.solver, ctx.state, ctx.dt, ctx.max_checkpoints = solver, state, float(dt), int(max_checkpoints)
        scale = np.exp(log_rate_scale.detach().to("cpu", torch.float64).numpy())
        solver.set_rate_scale(scale)
        _load(state, y0)
        solver.update_state_parameters(state)
        result = solver.solve(ctx.dt, state, method="fused", step_control="per_cell")
        if not result.converged:
            raise RuntimeError(f"solve did not converge: {result.state}")
        state.sync_outputs_to_host()
        ctx.save_for_backward(y0)
        return torch.as_tensor(state.concentrations(), dtype=torch.float64, device=y0.device)

    @staticmethod
    def backward(ctx, grad_y: torch.Tensor):
        (y0,) = ctx.saved_tensors
        solver, state = ctx.solver, ctx.state
        _load(state, y0)
        cols = solver.compiled.species_columns
        g = np.zeros((state.n_cells, state.S))
        g[:, cols] = grad_y.detach().to("cpu", torch.float64).numpy()
        dy0_cols, dlogk, _ = solver.solve_adjoint(ctx.dt, state, g, ctx.max_checkpoints)
        dy0 = torch.as_tensor(dy0_cols[:, cols], dtype=torch.float64, device=y0.device)
        dk = torch.as_tensor(dlogk, dtype=torch.float64, device=y0.device)
        return dy0, dk, None, None, None, None


def _load(state: State, y0: torch.Tensor):
    state.set_concentrations(y0.detach().to("cpu", torch.float64).numpy())
    state.sync_inputs_to_device()
