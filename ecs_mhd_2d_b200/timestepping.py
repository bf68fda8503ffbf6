"""Lawson integrating-factor steppers (reference: jax_scripts/lib/timestepping.py).

The reference steppers are generic in ``v_fn``/``L_diag``; here the MHD
right-hand side, its dissipation L_diag = dissipation(param_dict) and the
dealiasing mask are fused into the kernels, so ``param_dict`` replaces those
three arguments.
"""

from __future__ import annotations

import torch

from . import context as _ctx


def lawson_rk4(f, t, steps, param_dict):
    """Lawson-RK4 of the rfft2 state f [..., 2, n, n//2+1] over time t in `steps`
    steps with the mask applied to the integrating factor
    (timestepping.py:46-81 with v_fn = state_vel(., include_dissipation=False),
    L_diag = dissipation(param_dict), mask = param_dict["mask"])."""
    n = f.shape[-2]
    rdt = torch.float64 if f.dtype == torch.complex128 else torch.float32
    lead = f.shape[:-3]
    out = f.reshape(-1, 2, n, n // 2 + 1).contiguous().clone()
    B = out.shape[0]
    ctx = _ctx.get_context(param_dict, n, rdt, B)
    ctx.call("ecs_lawson_rk4", _ctx.ptr(out), float(t), int(steps), B, _ctx.stream_ptr())
    return out.reshape(*lead, 2, n, n // 2 + 1)
