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
    n = _ctx.check_spectral(f)
    rdt = torch.float64 if f.dtype == torch.complex128 else torch.float32
    lead = f.shape[:-3]
    out = f.reshape(-1, 2, n, n // 2 + 1).contiguous().clone()
    B = out.shape[0]
    if B == 0:
        return out.reshape(f.shape)
    ctx = _ctx.get_context(param_dict, n, rdt, B)
    ctx.call("ecs_lawson_rk4", _ctx.ptr(out), float(t), int(steps), B, _ctx.stream_ptr())
    return out.reshape(*lead, 2, n, n // 2 + 1)


def integrate(f, t, steps, param_dict, mode):
    """Fixed-step integration of the rfft2 state f [..., 2, n, n//2+1] over time
    t in `steps` steps in one of mismatch_RPO's fixed-step modes ("RK4",
    "Lawson_RK4", "Lawson_RK6", "TDRK4"; timestepping.py:17-149 with the v_fn,
    L_diag and mask of loss_functions.py:49-85).  Returns a new tensor."""
    from . import _lib
    codes = {"RK4": _lib.ECS_MODE_RK4, "Lawson_RK4": _lib.ECS_MODE_LAWSON_RK4,
             "Lawson_RK6": _lib.ECS_MODE_LAWSON_RK6, "TDRK4": _lib.ECS_MODE_TDRK4}
    if mode not in codes:
        raise ValueError(f"integrate: fixed-step mode expected, got {mode}")
    n = _ctx.check_spectral(f)
    rdt = torch.float64 if f.dtype == torch.complex128 else torch.float32
    lead = f.shape[:-3]
    out = f.reshape(-1, 2, n, n // 2 + 1).contiguous().clone()
    B = out.shape[0]
    if B == 0:
        return out.reshape(f.shape)
    ctx = _ctx.get_context(param_dict, n, rdt, B)
    ctx.call("ecs_integrate", codes[mode], _ctx.ptr(out), float(t), int(steps), B, _ctx.stream_ptr())
    return out.reshape(*lead, 2, n, n // 2 + 1)


def lawson_rk6(f, t, steps, param_dict):
    """Lawson sixth-order RK (timestepping.py:83-125), masked integrating factor."""
    return integrate(f, t, steps, param_dict, "Lawson_RK6")


def rk4(f, t, steps, param_dict):
    """Classic RK4 with dissipation in the right-hand side (timestepping.py:17-44)."""
    return integrate(f, t, steps, param_dict, "RK4")


def tdrk4(f, t, steps, param_dict):
    """Two-derivative RK4 (timestepping.py:127-149) with v_fn = state_vel(., include_dissipation=True)."""
    return integrate(f, t, steps, param_dict, "TDRK4")
