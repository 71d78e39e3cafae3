"""torch.autograd bridge for the Python assimilation utilities: J of a recorded trajectory as a
differentiable function of the per-cell friction coefficients, the bed and the initial state.

    J = replay_cost(model, friction_1=n, friction_2=n)   # sw2d_replay_cost
    J.backward()                                          # sw2d_adjoint -> n.grad

forward writes the given tensors into the model (sw2d_set_param / sw2d_set_trajectory_start)
and replays the recorded trajectory; backward runs the checkpointed reverse sweep on the GPU
(no re-recording: the dt sequence stays the one recorded).  Arguments left as None keep the
model's current values and get no gradient.  The model must not be changed between forward and
backward.  Tensors may live on any device; they cross the C ABI as host float64 arrays of
cell_nb values in the caller's numbering.
"""
from __future__ import annotations

import numpy as np
import torch

_NAMES = ("friction_1", "friction_2", "z_b", "h0", "q0", "r0")


def _host(t: torch.Tensor) -> np.ndarray:
    return t.detach().to("cpu", torch.float64).contiguous().numpy()


class ReplayCost(torch.autograd.Function):
    @staticmethod
    def forward(ctx, model, friction_1, friction_2, z_b, h0, q0, r0):
        args = dict(zip(_NAMES, (friction_1, friction_2, z_b, h0, q0, r0)))
        for name in ("friction_1", "friction_2", "z_b"):
            if args[name] is not None:
                model.set_param(name, _host(args[name]))
        if any(args[k] is not None for k in ("h0", "q0", "r0")):
            if not all(args[k] is not None for k in ("h0", "q0", "r0")):
                raise ValueError("h0, q0 and r0 are given together")
            model.set_trajectory_start(_host(h0), _host(q0), _host(r0))
        J = model.replay_cost()
        ctx.model = model
        ctx.given = [(name, t.device, t.dtype) if t is not None else None for name, t in args.items()]
        ref = next((t for t in args.values() if t is not None), None)
        device = ref.device if ref is not None else "cpu"
        return torch.tensor(J, dtype=torch.float64, device=device)

    @staticmethod
    def backward(ctx, gJ):
        wanted = [g[0] for g in ctx.given if g is not None]
        _, grads = ctx.model.adjoint(wrt=tuple(wanted))
        out = [None]
        for g in ctx.given:
            if g is None:
                out.append(None)
                continue
            name, device, dtype = g
            out.append(torch.from_numpy(grads[name]).to(device=device, dtype=dtype) * gJ.to(device=device, dtype=dtype))
        return tuple(out)


def replay_cost(model, friction_1=None, friction_2=None, z_b=None, h0=None, q0=None, r0=None) -> torch.Tensor:
    """J of the model's recorded trajectory, differentiable in the given tensors."""
    return ReplayCost.apply(model, friction_1, friction_2, z_b, h0, q0, r0)
