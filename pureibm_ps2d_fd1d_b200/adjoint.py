"""Differentiable drag objective: the engine's discrete adjoint behind a
torch.autograd.Function.

    from pureibm_ps2d_fd1d_b200 import config
    from pureibm_ps2d_fd1d_b200.adjoint import drag_objective
    prm, xc = config.adjoint_case()                  # 96^3, 30 spheres, SET_MPG, fixed dt
    state = ...                                      # initial state (Solver.get_state())
    x = torch.tensor(xc, requires_grad=True)
    g = torch.tensor(prm["mpg"], requires_grad=True)
    J = drag_objective(x, g, prm, state, nsteps=200)
    J.backward()                                     # x.grad = dJ/dxc, g.grad = dJ/dmpg

J = (1/K) sum_{n=1..K} e . sum_m (pres_m + visc_m): the summed pressure +
viscous surface force of calc_pres_visc_drag (boundary_condition.F90:
1481-1645) inside each of the K steps, projected on e.  When a gradient is
requested, the forward call runs pibm_adjoint_run (K steps with checkpoints,
then the reverse sweep) and backward returns the stored gradients scaled by
the incoming gradient; otherwise only the K forward steps run.  Torch is used
for the autograd plumbing only: both sweeps are the engine's CUDA kernels.
"""
from __future__ import annotations

import numpy as np
import torch

from . import Solver, config


def _solver(params: dict, xc: np.ndarray, mpg: np.ndarray, state: dict) -> Solver:
    p = dict(params)
    p["mpg"] = tuple(float(v) for v in mpg)
    s = Solver(config.make_params(p), xc)
    st = dict(state)
    st["mpg"] = np.asarray(mpg, dtype=np.float64)
    s.set_state(st)
    return s


class DragObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xc, mpg, params, state, nsteps, direction, checkpoint_every):
        x = xc.detach().to("cpu", torch.float64).numpy()
        g = mpg.detach().to("cpu", torch.float64).numpy()
        e = np.asarray(direction, dtype=np.float64)
        s = _solver(params, x, g, state)
        try:
            if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
                out = s.adjoint(int(nsteps), e, int(checkpoint_every))
                J = out["J"]
                ctx.save_for_backward(torch.as_tensor(out["g_xc"]).to(xc.device), torch.as_tensor(out["g_mpg"]).to(mpg.device))
            else:
                J = 0.0
                for _ in range(int(nsteps)):
                    r = s.step(1)
                    J += float(np.dot(e, np.asarray(r["visc_total"]) - np.asarray(r["pres_total"])))
                J /= int(nsteps)
        finally:
            s.close()
        return torch.tensor(J, dtype=torch.float64, device=xc.device)

    @staticmethod
    def backward(ctx, grad_J):
        g_xc, g_mpg = ctx.saved_tensors
        return grad_J * g_xc, grad_J * g_mpg, None, None, None, None, None


def drag_objective(xc: torch.Tensor, mpg: torch.Tensor, params: dict, state: dict, nsteps: int,
                   direction=(1.0, 0.0, 0.0), checkpoint_every: int = 20) -> torch.Tensor:
    """J(xc, mpg) as a differentiable scalar (see the module docstring).
    xc: (nbody, 3) sphere centres in grid units; mpg: (3,) imposed mean
    pressure gradient; params: a config dict with SET_MPG and a fixed dt;
    state: the initial state of the K steps."""
    return DragObjective.apply(xc, mpg, params, state, nsteps, tuple(direction), checkpoint_every)
