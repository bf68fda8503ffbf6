"""Tangent (JVP) and adjoint (VJP) of the RPO objective through the C-ABI.

The reference obtains these with jax.jvp / jax.vjp of objective_RPO
(jax_scripts/lib/utils.py:93-119, jax_scripts/newton.py:165-170) and
jax.value_and_grad of loss_RPO (jax_scripts/adjoint_descent.py:90-91).  Here a
primal point is *linearised* once (forward solve with a trajectory record kept
on the device) and any number of tangents / cotangents are then pushed through
hand-written tangent and adjoint kernels, batched.
"""

from __future__ import annotations

import torch

from . import _lib
from . import context as _ctx
from .loss_functions import _empty_like_out, grid_of, objective_RPO, prep_inputs, shoot_cfg


class Objective:
    """objective_RPO(input_dict, param_dict, mode) as a callable with cached
    linearisations for jvp / vjp."""

    def __init__(self, param_dict, mode, ctx=None):
        """`ctx` pins a private context (e.g. one per serving worker thread);
        by default contexts come from the shared per-physics cache."""
        self.param_dict, self.mode = param_dict, mode
        self.cfg = shoot_cfg(param_dict, mode)
        self._key = None
        self._ctx = None
        self._own_ctx = ctx
        self.last_info = None
        self.last_value = None

    def __call__(self, input_dict):
        return objective_RPO(input_dict, self.param_dict, self.mode)

    # -- linearisation -------------------------------------------------
    def _primal_key(self, fields, T, sx):
        return (fields.data_ptr(), fields._version, tuple(fields.shape), fields.dtype, float(T), float(sx))

    def linearize(self, input_dict, force=False, batch=1):
        """Primal solve with trajectory record; `batch` sizes the workspace for the
        tangent/cotangent batches that follow (growing it later drops the record)."""
        fields, T, sx, batched = prep_inputs(input_dict)
        if fields.shape[0] != 1:
            raise ValueError("linearize takes one primal point")
        n = fields.shape[-1]
        if self._own_ctx is not None:
            ctx = self._own_ctx
            ctx.ensure_batch(batch)
        else:
            ctx = _ctx.get_context(self.param_dict, n, fields.dtype, batch)
        key = (ctx.generation,) + self._primal_key(input_dict["fields"]
                                                                                    if isinstance(input_dict["fields"], torch.Tensor)
                                                                                    else fields, T[0], sx[0])
        if not force and key == self._key and self._ctx is ctx:
            return ctx
        out = torch.empty_like(fields)
        info = _lib.EcsInfo()
        ctx.call("ecs_linearize", self.cfg, _ctx.ptr(fields), _ctx.ptr(T), _ctx.ptr(sx), _ctx.ptr(out), info,
                 _ctx.stream_ptr())
        self._key, self._ctx = key, ctx
        self._fields_ref = (fields, T, sx)   # keep the primal alive while the key is cached
        self.last_value = {"fields": out[0], "T": torch.zeros((), dtype=torch.float64, device=out.device),
                           "sx": torch.zeros((), dtype=torch.float64, device=out.device)}
        self.last_info = {"completed": bool(info.completed), "s": info.s, "accepted": info.accepted,
                          "rejected": info.rejected, "fevals": info.fevals}
        return ctx

    def linearize_jvp(self, primal_dict, tangent_dict):
        """Objective value and tangents in one call (jax.jvp(obj, (x,), (v,)),
        jax_scripts/lib/utils.py:108): the primal solve is re-run with its
        record and overlapped with the tangent sweep (ecs_linearize_jvp); the
        linearisation is kept for later jvp / vjp calls.  Returns (value, jvp)."""
        fields, T, sx, _ = prep_inputs(primal_dict)
        if fields.shape[0] != 1:
            raise ValueError("linearize_jvp takes one primal point")
        dfields, dT, dsx, batched = prep_inputs(tangent_dict, n=fields.shape[-1], dtype=fields.dtype,
                                                what="tangent fields")
        B, n = dfields.shape[0], fields.shape[-1]
        if B == 0:
            self.linearize(primal_dict)
            return self.last_value, _empty_like_out(dfields)
        if self._own_ctx is not None:
            ctx = self._own_ctx
            ctx.ensure_batch(B)
        else:
            ctx = _ctx.get_context(self.param_dict, n, fields.dtype, B)
        out = torch.empty_like(fields)
        info = _lib.EcsInfo()
        dout = torch.empty_like(dfields)
        oT = torch.empty(B, dtype=torch.float64, device=dfields.device)
        osx = torch.empty(B, dtype=torch.float64, device=dfields.device)
        ctx.call("ecs_linearize_jvp", self.cfg, _ctx.ptr(fields), _ctx.ptr(T), _ctx.ptr(sx), _ctx.ptr(out), info,
                 _ctx.ptr(dfields), _ctx.ptr(dT), _ctx.ptr(dsx), _ctx.ptr(dout), _ctx.ptr(oT), _ctx.ptr(osx), B,
                 _ctx.stream_ptr())
        key = (ctx.generation,) + self._primal_key(
            primal_dict["fields"] if isinstance(primal_dict["fields"], torch.Tensor) else fields, T[0], sx[0])
        self._key, self._ctx = key, ctx
        self._fields_ref = (fields, T, sx)
        zero = torch.zeros((), dtype=torch.float64, device=out.device)
        self.last_value = {"fields": out[0], "T": zero, "sx": zero.clone()}
        self.last_info = {"completed": bool(info.completed), "s": info.s, "accepted": info.accepted,
                          "rejected": info.rejected, "fevals": info.fevals}
        tan = {"fields": dout, "T": oT, "sx": osx} if batched else {"fields": dout[0], "T": oT[0], "sx": osx[0]}
        return self.last_value, tan

    def jvp(self, primal_dict, tangent_dict):
        """Tangent of objective_RPO at primal_dict; tangent_dict may carry a leading batch dim."""
        n, dtype = grid_of(primal_dict)
        dfields, dT, dsx, batched = prep_inputs(tangent_dict, n=n, dtype=dtype, what="tangent fields")
        B = dfields.shape[0]
        if B == 0:
            return _empty_like_out(dfields)
        ctx = self.linearize(primal_dict, batch=B)
        out = torch.empty_like(dfields)
        oT = torch.empty(B, dtype=torch.float64, device=dfields.device)
        osx = torch.empty(B, dtype=torch.float64, device=dfields.device)
        ctx.call("ecs_jvp", _ctx.ptr(dfields), _ctx.ptr(dT), _ctx.ptr(dsx), _ctx.ptr(out), _ctx.ptr(oT), _ctx.ptr(osx),
                 B, _ctx.stream_ptr())
        if not batched:
            return {"fields": out[0], "T": oT[0], "sx": osx[0]}
        return {"fields": out, "T": oT, "sx": osx}


def _as_objective(obj, param_dict):
    if isinstance(obj, Objective):
        return obj
    if isinstance(obj, str):
        return Objective(param_dict, obj)
    raise TypeError("obj must be an Objective or a mode string (e.g. 'Lawson_RK4', 'TDRK4')")


def compile_objective_and_Jacobian(input_dict, param_dict, obj):
    """(objective, jac) as in utils.compile_objective_and_Jacobian
    (jax_scripts/lib/utils.py:93-119); jac(primal, tangent) is the JVP."""
    o = _as_objective(obj, param_dict)
    o.linearize(input_dict)
    return o, o.jvp


def _vjp_call(obj, primal_dict, cot):
    n, dtype = grid_of(primal_dict)
    cf, cT, csx, batched = prep_inputs(cot, n=n, dtype=dtype, what="cotangent fields")
    B = cf.shape[0]
    if B == 0:
        return _empty_like_out(cf)
    ctx = obj.linearize(primal_dict, batch=B)
    g = torch.empty_like(cf)
    gT = torch.empty(B, dtype=torch.float64, device=cf.device)
    gsx = torch.empty(B, dtype=torch.float64, device=cf.device)
    ctx.call("ecs_vjp", _ctx.ptr(cf), _ctx.ptr(cT), _ctx.ptr(csx), _ctx.ptr(g), _ctx.ptr(gT), _ctx.ptr(gsx), B,
             _ctx.stream_ptr())
    if not batched:
        return {"fields": g[0], "T": gT[0], "sx": gsx[0]}
    return {"fields": g, "T": gT, "sx": gsx}


def vjp(obj, primal_dict):
    """(out, jacT) like jax.vjp(obj, input_dict) (jax_scripts/newton.py:168):
    jacT(cotangent_dict) -> (grad_dict,).  Cotangents may carry a batch dim."""
    obj = obj if isinstance(obj, Objective) else Objective(*obj)
    obj.linearize(primal_dict)
    out = obj.last_value

    def jacT(cot):
        return (_vjp_call(obj, primal_dict, cot),)

    return out, jacT


def loss_and_grad(input_dict, param_dict, mode, normalized=False, obj=None, ctx=None):
    """((loss, info), grad) of loss_RPO = mean(irfft2(f - f0)^2) (jax_scripts/lib/loss_functions.py:99-111)
    as jax.value_and_grad(..., has_aux=True) gives it (jax_scripts/adjoint_descent.py:90-96).
    normalized=True uses |shift(u(T)) - u(0)|^2 / |u(0)|^2 instead."""
    obj = obj or Objective(param_dict, mode, ctx=ctx)
    obj._key = None   # the loss is evaluated at a new point each call
    ctx = obj.linearize(input_dict)
    out = obj.last_value["fields"]
    n = out.shape[-1]
    cnt = 2 * n * n
    loss = torch.sum(out.double() ** 2) / cnt
    cot = {"fields": (out / (n * n)).contiguous(), "T": 0.0, "sx": 0.0}
    g = _vjp_call(obj, input_dict, cot)
    if normalized:
        u0 = prep_inputs(input_dict)[0][0]
        nu0 = torch.sum(u0.double() ** 2)
        num = torch.sum(out.double() ** 2)
        lossn = num / nu0
        scale = cnt / nu0
        g = {"fields": g["fields"] * scale - (2 * lossn / nu0) * u0, "T": g["T"] * scale, "sx": g["sx"] * scale}
        loss = lossn
    return (loss, obj.last_info), g


class LossRPOFunction(torch.autograd.Function):
    """loss_RPO as a differentiable torch op whose backward is the hand-written
    adjoint Lawson-RK kernel (checkpointing is inside the linearisation)."""

    @staticmethod
    def forward(ctx, fields, T, sx, param_dict, mode, normalized):
        (loss, info), g = loss_and_grad({"fields": fields.detach(), "T": T.detach(), "sx": sx.detach()},
                                        param_dict, mode, normalized)
        ctx.save_for_backward(g["fields"], g["T"].reshape(()), g["sx"].reshape(()))
        return loss

    @staticmethod
    def backward(ctx, gout):
        gf, gT, gsx = ctx.saved_tensors
        return gout * gf, gout * gT.to(gout.dtype), gout * gsx.to(gout.dtype), None, None, None


def loss_rpo_autograd(fields, T, sx, param_dict, mode, normalized=False):
    return LossRPOFunction.apply(fields, T, sx, param_dict, mode, normalized)
