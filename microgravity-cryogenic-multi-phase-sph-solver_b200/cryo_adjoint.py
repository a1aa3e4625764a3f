"""Differentiable windows of the solver: a torch.autograd.Function over the
hand-written adjoint of the step.

`slosh_window(solver, sigma, contact_angle, lee, knots, steps)` runs `steps`
steps of a CryoSPH.Solver from its current state with

  sigma          surface tension coefficient (FluidProperties.sigma)
  contact_angle  static contact angle in degrees (SolverConfig.contact_angle_deg)
  lee            Lee coefficient, evaporation and condensation alike (1/s)
  knots          (K, 3) frame accelerations, piecewise constant over K equal
                 parts of the window (a ManeuverProfile with short ramps
                 placed between steps, so every step sees exactly one knot)

and returns the tensor [time-integrated slosh force (3), time-integrated
slosh moment (3), ullage pressure after the last step].  Its backward runs
the reverse passes of every step (CryoSPH.Solver.adjoint_backward): the
window is recomputed from state checkpoints taken every `checkpoint_every`
steps, and the neighbour sets, phases and branch decisions of each step are
those of the forward run.  The solver is left in the window's final state.

The solver must use a fixed time step, a pinned sound speed and particles
that neither split nor merge inside the window (split_ratio large,
merge_ratio 0); the adjoint entry points reject other configurations.
"""
from __future__ import annotations

import numpy as np
import torch

import CryoSPH as cs


def knot_schedule(t_start: float, dt: float, steps: int, nknots: int):
    """The ManeuverProfile of piecewise-constant knots over a window of
    `steps` steps of size dt starting at t_start, and the knot each step
    sees.  A step's frame is evaluated at the end of the step
    (sph_solver.cu:516-521); the ramps between knots lie strictly between
    two such evaluation times."""
    if nknots < 1 or nknots > steps:
        raise ValueError("need 1 <= knots <= steps")
    bounds = [round(k * steps / nknots) for k in range(nknots + 1)]
    times = []
    seg = np.empty(steps, np.int64)
    for k in range(nknots):
        n0, n1 = bounds[k], bounds[k + 1]
        seg[n0:n1] = k
        start = t_start if k == 0 else t_start + (n0 + 0.75) * dt
        end = t_start + (n1 + 0.25) * dt
        times += [start, end]
    return np.asarray(times, np.float64), seg


def _maneuver(times, knots_np):
    acc = np.repeat(np.asarray(knots_np, np.float64), 2, axis=0)
    return cs.ManeuverProfile([float(t) for t in times], acc)


class SloshWindow(torch.autograd.Function):
    """Forward: one differentiated window (see the module docstring).
    Backward: the hand-written reverse sweep; gradients for sigma,
    contact_angle, lee and knots."""

    @staticmethod
    def forward(ctx, sigma, contact_angle, lee, knots, solver, steps, checkpoint_every):
        dt = float(solver.config.fixed_dt)
        times, seg = knot_schedule(solver.time, dt, int(steps), int(knots.shape[0]))
        solver.set_surface_tension(float(sigma))
        solver.set_contact_angle(float(contact_angle))
        solver.set_lee_coefficients(float(lee), float(lee))
        solver.set_maneuver(_maneuver(times, knots.detach().cpu().numpy()))
        obj = solver.adjoint_forward(int(steps), int(checkpoint_every))
        ctx.solver = solver
        ctx.seg = torch.as_tensor(seg)
        ctx.nknots = int(knots.shape[0])
        ctx.dtype = knots.dtype
        return torch.as_tensor(obj, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad):
        seed = grad.detach().to(torch.float64).cpu().numpy()
        g = ctx.solver.adjoint_backward([float(v) for v in seed])
        fa = torch.as_tensor(g["frame_acceleration"], dtype=torch.float64)
        gk = torch.zeros(ctx.nknots, 3, dtype=torch.float64).index_add_(0, ctx.seg, fa)
        t = lambda v: torch.tensor(v, dtype=torch.float64)
        return (t(g["sigma"]), t(g["contact_angle"]), t(g["lee_evaporation"] + g["lee_condensation"]),
                gk.to(ctx.dtype), None, None, None)


def slosh_window(solver, sigma, contact_angle, lee, knots, steps, checkpoint_every=20):
    """[int F (3), int M (3), p_ullage] of a differentiated window."""
    as_t = lambda v: v if torch.is_tensor(v) else torch.tensor(float(v), dtype=torch.float64)
    knots = knots if torch.is_tensor(knots) else torch.as_tensor(np.asarray(knots, np.float64))
    return SloshWindow.apply(as_t(sigma), as_t(contact_angle), as_t(lee), knots, solver, int(steps),
                             int(checkpoint_every))
