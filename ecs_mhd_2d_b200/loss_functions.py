"""RPO shooting objective and loss (reference: jax_scripts/lib/loss_functions.py).

Inputs follow the reference's dict layout ``{"fields": real[2,n,n], "T": (),
"sx": ()}``; a leading batch dimension ([B,2,n,n], [B], [B]) evaluates B
candidates in one set of launches.
"""

from __future__ import annotations

import torch

from . import _lib
from . import context as _ctx

MODES = {"Lawson_RK4": _lib.ECS_MODE_LAWSON_RK4, "Lawson_RK43": _lib.ECS_MODE_LAWSON_RK43,
         "RK4": _lib.ECS_MODE_RK4, "Lawson_RK6": _lib.ECS_MODE_LAWSON_RK6, "TDRK4": _lib.ECS_MODE_TDRK4}


def shoot_cfg(param_dict, mode):
    """ecs_shoot_cfg from param_dict (loss_functions.py:48-94)."""
    if mode not in MODES:
        # loss_functions.py:86-88 prints and exits; here it is an exception
        raise ValueError(f"You selected mode = {mode}, which does not exist.")
    c = _lib.EcsShootCfg()
    c.mode = MODES[mode]
    c.num_checkpoints = int(param_dict.get("num_checkpoints", 1))
    c.ministeps = int(param_dict.get("ministeps", param_dict.get("steps", 1)))
    if mode == "Lawson_RK6":   # one run of param_dict["steps"] steps over T (loss_functions.py:66-71)
        c.num_checkpoints, c.ministeps = 1, int(param_dict["steps"])
    c.shift_reflect_ny = int(param_dict.get("shift_reflect_ny", 0))
    c.rot = int(bool(param_dict.get("rot", False)))
    ad = param_dict.get("adaptive_dict", {}) or {}
    c.atol = float(ad.get("atol", 1e-4))
    c.h0 = float(ad.get("h0", 1e-2))
    c.max_steps_per_checkpoint = int(ad.get("max_steps_per_checkpoint", 1024))
    c.checkpoints = int(ad.get("checkpoints", 1))
    c.ckpt_every = int(param_dict.get("ckpt_every", 0))
    for name in ("num_checkpoints", "ministeps", "checkpoints", "max_steps_per_checkpoint"):
        if getattr(c, name) < 1:
            raise ValueError(f"{name} must be >= 1, got {getattr(c, name)}")
    if c.ckpt_every < 0:
        raise ValueError(f"ckpt_every must be >= 0, got {c.ckpt_every}")
    return c


def prep_inputs(input_dict, n=None, dtype=None, what="fields"):
    """Batched, contiguous device tensors (fields [B,2,n,n], T [B], sx [B]) and
    whether the input carried a batch dimension.  The shapes are checked on the
    host first: fields [2, n, n] or [B, 2, n, n] (side `n` when given, e.g. a
    tangent's against its primal), T and sx one value or B values.  `dtype`
    converts the fields (a tangent takes its primal's precision)."""
    f = input_dict["fields"]
    if not isinstance(f, torch.Tensor):
        f = torch.as_tensor(f)
    _ctx.check_fields(f, what, n)
    batched = f.dim() == 4
    fb = (f if batched else f.unsqueeze(0))
    if dtype is not None:
        fb = fb.to(dtype)
    elif fb.dtype not in (torch.float64, torch.float32):
        fb = fb.to(torch.float64)
    B = fb.shape[0]

    def scal(v, name):
        t = torch.as_tensor(v, dtype=torch.float64).reshape(-1)
        if t.numel() != B and t.numel() != 1:
            raise ValueError(f"{name} has {t.numel()} values for a batch of {B}")
        return t

    def dev(t):
        t = t.to("cuda")
        return (t.expand(B) if t.numel() == 1 and B != 1 else t).contiguous()

    T, sx = scal(input_dict["T"], "T"), scal(input_dict["sx"], "sx")   # both checked before any copy
    return fb.to("cuda").contiguous(), dev(T), dev(sx), batched


def grid_of(input_dict):
    """(n, dtype) that prep_inputs gives the fields of input_dict, without copying them."""
    f = input_dict["fields"]
    if not isinstance(f, torch.Tensor):
        f = torch.as_tensor(f)
    _ctx.check_fields(f)
    return f.shape[-1], (f.dtype if f.dtype in (torch.float64, torch.float32) else torch.float64)


def _empty_like_out(fields):
    z = torch.empty(0, dtype=torch.float64, device=fields.device)
    return {"fields": torch.empty_like(fields), "T": z, "sx": z.clone()}


def objective_RPO(input_dict, param_dict, mode, ctx=None):
    """{"fields": irfft2(f0 - g.Phi_T(f0)), "T": pt, "sx": px} (loss_functions.py:132-148).
    pt and px are phase conditions whose value is exactly 0 (:128-129).
    `ctx` pins a private context (e.g. a serving worker thread's); by default
    the shared per-physics context."""
    cfg = shoot_cfg(param_dict, mode)
    fields, T, sx, batched = prep_inputs(input_dict)
    B, n = fields.shape[0], fields.shape[-1]
    if B == 0:
        return _empty_like_out(fields)
    if ctx is None:
        ctx = _ctx.get_context(param_dict, n, fields.dtype, B)
    else:
        ctx.ensure_batch(B)
    out = torch.empty_like(fields)
    oT = torch.empty(B, dtype=torch.float64, device=fields.device)
    osx = torch.empty(B, dtype=torch.float64, device=fields.device)
    info = (_lib.EcsInfo * B)()
    ctx.call("ecs_objective", cfg, _ctx.ptr(fields), _ctx.ptr(T), _ctx.ptr(sx), _ctx.ptr(out),
             _ctx.ptr(oT), _ctx.ptr(osx), info, B, _ctx.stream_ptr())
    if not batched:
        return {"fields": out[0], "T": oT[0], "sx": osx[0]}
    return {"fields": out, "T": oT, "sx": osx}


def loss_RPO(input_dict, param_dict, mode):
    """(mean(irfft2(f - f0)^2), info) (loss_functions.py:99-111)."""
    cfg = shoot_cfg(param_dict, mode)
    fields, T, sx, batched = prep_inputs(input_dict)
    B, n = fields.shape[0], fields.shape[-1]
    if B == 0:
        return torch.empty(0, dtype=torch.float64, device=fields.device), []
    ctx = _ctx.get_context(param_dict, n, fields.dtype, B)
    loss = torch.empty(B, dtype=torch.float64, device=fields.device)
    info = (_lib.EcsInfo * B)()
    ctx.call("ecs_loss", cfg, _ctx.ptr(fields), _ctx.ptr(T), _ctx.ptr(sx), _ctx.ptr(loss), info, B,
             _ctx.stream_ptr())
    infos = [{"completed": bool(i.completed), "s": i.s, "accepted": i.accepted, "rejected": i.rejected,
              "fevals": i.fevals} for i in info]
    if not batched:
        return loss[0], infos[0]
    return loss, infos


def dealias(fields, param_dict):
    """irfft2(mask * rfft2(fields)) (newton.py:211-214, adjoint_descent.py:111-114)."""
    _ctx.check_fields(fields)
    f = fields if fields.dim() == 4 else fields.unsqueeze(0)
    f = f.contiguous()
    B, n = f.shape[0], f.shape[-1]
    if B == 0:
        return torch.empty_like(fields)
    ctx = _ctx.get_context(param_dict, n, f.dtype, B)
    out = torch.empty_like(f)
    ctx.call("ecs_dealias", _ctx.ptr(f), _ctx.ptr(out), B, _ctx.stream_ptr())
    return out if fields.dim() == 4 else out[0]
