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
from .loss_functions import _empty_like_out, grid_of, loss_RPO, objective_RPO, prep_inputs, shoot_cfg


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
        self._token = None
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
        if not force and key == self._key and self._ctx is ctx and ctx.lin_token is self._token:
            return ctx
        out = torch.empty_like(fields)
        info = _lib.EcsInfo()
        ctx.lin_token = None
        ctx.call("ecs_linearize", self.cfg, _ctx.ptr(fields), _ctx.ptr(T), _ctx.ptr(sx), _ctx.ptr(out), info,
                 _ctx.stream_ptr())
        self._key, self._ctx = key, ctx
        self._token = ctx.lin_token = object()
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
        ctx.lin_token = None
        ctx.call("ecs_linearize_jvp", self.cfg, _ctx.ptr(fields), _ctx.ptr(T), _ctx.ptr(sx), _ctx.ptr(out), info,
                 _ctx.ptr(dfields), _ctx.ptr(dT), _ctx.ptr(dsx), _ctx.ptr(dout), _ctx.ptr(oT), _ctx.ptr(osx), B,
                 _ctx.stream_ptr())
        key = (ctx.generation,) + self._primal_key(
            primal_dict["fields"] if isinstance(primal_dict["fields"], torch.Tensor) else fields, T[0], sx[0])
        self._key, self._ctx = key, ctx
        self._token = ctx.lin_token = object()
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


def jvp_multi(primals, tangents, param_dicts, mode="Lawson_RK4", ctx=None):
    """Objectives and one JVP each for several candidates in one device sweep:
    [jax.jvp(obj_b, (x_b,), (v_b,)) for each b] (jax_scripts/lib/utils.py:108,
    one call per candidate's Arnoldi step, jax_scripts/newton.py:165), batched
    across candidates (ecs_jvp_multi; Lawson_RK4 only, forward mode, nothing
    kept).  `primals`, `tangents` and `param_dicts` are lists of equal length;
    the param dicts share the grid, dtype and physics (nu, eta, b0, forcing) and
    may differ in num_checkpoints, ministeps, shift_reflect_ny and rot.
    Returns (values, jvps), lists of {"fields", "T", "sx"} dicts."""
    if mode != "Lawson_RK4":
        raise ValueError(f"jvp_multi runs Lawson_RK4, got {mode}")
    if not (len(primals) == len(tangents) == len(param_dicts)):
        raise ValueError("jvp_multi: primals, tangents and param_dicts differ in length")
    B = len(primals)
    if B == 0:
        return [], []
    xs = [prep_inputs(p) for p in primals]
    n, dtype = xs[0][0].shape[-1], xs[0][0].dtype
    for (f, _, _, _) in xs:
        if f.shape != (1, 2, n, n) or f.dtype != dtype:
            raise ValueError("jvp_multi: every primal is one state of the same grid and dtype")
    ts = [prep_inputs(t, n=n, dtype=dtype, what="tangent fields") for t in tangents]
    for (f, _, _, _) in ts:
        if f.shape[0] != 1:
            raise ValueError("jvp_multi: one tangent per candidate")
    key = _ctx.physics_key(param_dicts[0])
    if any(_ctx.physics_key(pd) != key for pd in param_dicts[1:]):
        raise ValueError("jvp_multi: the candidates' param dicts differ in grid or physics")
    cfgs = (_lib.EcsShootCfg * B)()
    for b, pd in enumerate(param_dicts):
        cfgs[b] = shoot_cfg(pd, mode)
    if ctx is None:
        ctx = _ctx.get_context(param_dicts[0], n, dtype, B)
    else:
        ctx.ensure_batch(B)
    fields = torch.cat([x[0] for x in xs]).contiguous()
    T = torch.cat([x[1] for x in xs]).contiguous()
    sx = torch.cat([x[2] for x in xs]).contiguous()
    dfields = torch.cat([t[0] for t in ts]).contiguous()
    dT = torch.cat([t[1] for t in ts]).contiguous()
    dsx = torch.cat([t[2] for t in ts]).contiguous()
    out = torch.empty_like(fields)
    dout = torch.empty_like(dfields)
    oT = torch.empty(B, dtype=torch.float64, device=fields.device)
    osx = torch.empty(B, dtype=torch.float64, device=fields.device)
    ctx.call("ecs_jvp_multi", cfgs, _ctx.ptr(fields), _ctx.ptr(T), _ctx.ptr(sx), _ctx.ptr(out), _ctx.ptr(dfields),
             _ctx.ptr(dT), _ctx.ptr(dsx), _ctx.ptr(dout), _ctx.ptr(oT), _ctx.ptr(osx), B, _ctx.stream_ptr())
    zero = torch.zeros((), dtype=torch.float64, device=fields.device)
    values = [{"fields": out[b], "T": zero, "sx": zero} for b in range(B)]
    jvps = [{"fields": dout[b], "T": oT[b], "sx": osx[b]} for b in range(B)]
    return values, jvps


def loss_grad_multi(inputs, param_dicts, mode="Lawson_RK4", ctx=None):
    """loss_RPO and its gradient for several candidates in one device sweep:
    [jax.value_and_grad(loss_RPO)(x_b) for each b] (jax_scripts/adjoint_descent.py:91,
    loss_functions.py:99-111), batched across candidates (ecs_loss_grad_multi;
    Lawson_RK4 only).  The param dicts share the grid, dtype and physics and may
    differ in num_checkpoints, ministeps, shift_reflect_ny and rot.  Returns a
    list of (loss, grad) with grad a {"fields", "T", "sx"} dict."""
    if mode != "Lawson_RK4":
        raise ValueError(f"loss_grad_multi runs Lawson_RK4, got {mode}")
    if len(inputs) != len(param_dicts):
        raise ValueError("loss_grad_multi: inputs and param_dicts differ in length")
    B = len(inputs)
    if B == 0:
        return []
    xs = [prep_inputs(x) for x in inputs]
    n, dtype = xs[0][0].shape[-1], xs[0][0].dtype
    for (f, _, _, _) in xs:
        if f.shape != (1, 2, n, n) or f.dtype != dtype:
            raise ValueError("loss_grad_multi: every input is one state of the same grid and dtype")
    key = _ctx.physics_key(param_dicts[0])
    if any(_ctx.physics_key(pd) != key for pd in param_dicts[1:]):
        raise ValueError("loss_grad_multi: the candidates' param dicts differ in grid or physics")
    cfgs = (_lib.EcsShootCfg * B)()
    for b, pd in enumerate(param_dicts):
        cfgs[b] = shoot_cfg(pd, mode)
    if ctx is None:
        ctx = _ctx.get_context(param_dicts[0], n, dtype, B)
    else:
        ctx.ensure_batch(B)
    fields = torch.cat([x[0] for x in xs]).contiguous()
    T = torch.cat([x[1] for x in xs]).contiguous()
    sx = torch.cat([x[2] for x in xs]).contiguous()
    loss = torch.empty(B, dtype=torch.float64, device=fields.device)
    g = torch.empty_like(fields)
    gT = torch.empty(B, dtype=torch.float64, device=fields.device)
    gsx = torch.empty(B, dtype=torch.float64, device=fields.device)
    ctx.call("ecs_loss_grad_multi", cfgs, _ctx.ptr(fields), _ctx.ptr(T), _ctx.ptr(sx), _ctx.ptr(loss), _ctx.ptr(g),
             _ctx.ptr(gT), _ctx.ptr(gsx), B, _ctx.stream_ptr())
    return [(loss[b], {"fields": g[b], "T": gT[b], "sx": gsx[b]}) for b in range(B)]


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


def _loss_of_residual(out, u0, normalized):
    """loss_RPO from the objective residual out = irfft2(f0 - f): mean(out^2)
    over the 2 n^2 entries (loss_functions.py:99-111), or with normalized=True
    |shift(u(T)) - u(0)|^2 / |u(0)|^2."""
    n = out.shape[-1]
    num = torch.sum(out.double() ** 2)
    if normalized:
        return num / torch.sum(u0.double() ** 2)
    return num / (2 * n * n)


def _loss_gradient(obj, input_dict, out, u0, normalized, gout=None):
    """Gradient of the loss (scaled by gout, the upstream gradient) through one
    adjoint sweep at obj's linearisation: the cotangent of the residual is
    d loss / d out = 2 out / (2 n^2), or 2 out / |u0|^2 normalised, plus, for
    the normalised loss, the explicit -2 loss u0 / |u0|^2 of its denominator."""
    n = out.shape[-1]
    cnt = 2 * n * n
    w = out / (n * n)
    if gout is not None:
        w = w * gout.to(out.dtype)
    g = _vjp_call(obj, input_dict, {"fields": w.contiguous(), "T": 0.0, "sx": 0.0})
    if not normalized:
        return g
    nu0 = torch.sum(u0.double() ** 2)
    lossn = torch.sum(out.double() ** 2) / nu0
    scale = cnt / nu0
    corr = (2 * lossn / nu0) * u0
    if gout is not None:
        corr = corr * gout
    return {"fields": g["fields"] * scale - corr, "T": g["T"] * scale, "sx": g["sx"] * scale}


def loss_and_grad(input_dict, param_dict, mode, normalized=False, obj=None, ctx=None):
    """((loss, info), grad) of loss_RPO = mean(irfft2(f - f0)^2) (jax_scripts/lib/loss_functions.py:99-111)
    as jax.value_and_grad(..., has_aux=True) gives it (jax_scripts/adjoint_descent.py:90-96).
    normalized=True uses |shift(u(T)) - u(0)|^2 / |u(0)|^2 instead."""
    obj = obj or Objective(param_dict, mode, ctx=ctx)
    obj._key = None   # the loss is evaluated at a new point each call
    obj.linearize(input_dict)
    out = obj.last_value["fields"]
    u0 = prep_inputs(input_dict)[0][0]
    loss = _loss_of_residual(out, u0, normalized)
    g = _loss_gradient(obj, input_dict, out, u0, normalized)
    return (loss, obj.last_info), g


class LossRPOFunction(torch.autograd.Function):
    """loss_RPO as a differentiable torch op.  forward runs the primal solve and
    keeps its trajectory record (checkpointed every ckpt_every steps when the
    param_dict asks for it); backward runs the hand-written adjoint Lawson-RK
    sweep over that record, with the upstream gradient folded into the
    cotangent.  When no gradient is wanted (``obj`` None: grad mode off or no
    input requiring grad) forward is the plain shooting, with no record."""

    @staticmethod
    def forward(ctx, fields, T, sx, param_dict, mode, normalized, obj):
        inp = {"fields": fields.detach(), "T": T.detach(), "sx": sx.detach()}
        u0 = fields.detach()
        if obj is None:
            loss, _ = loss_RPO(inp, param_dict, mode)
            if normalized:
                n = u0.shape[-1]
                loss = loss * (2 * n * n) / torch.sum(u0.double() ** 2)
            return loss
        obj._key = None
        obj.linearize(inp)
        out = obj.last_value["fields"]
        ctx.obj, ctx.inp, ctx.normalized = obj, inp, normalized
        ctx.save_for_backward(out, u0)
        return _loss_of_residual(out, u0, normalized)

    @staticmethod
    def backward(ctx, gout):
        out, u0 = ctx.saved_tensors
        g = _loss_gradient(ctx.obj, ctx.inp, out, u0, ctx.normalized, gout=gout)
        gT = g["T"].reshape(()).to(gout.dtype)
        gsx = g["sx"].reshape(()).to(gout.dtype)
        return g["fields"], gT, gsx, None, None, None, None


def loss_rpo_autograd(fields, T, sx, param_dict, mode, normalized=False):
    """loss_RPO(fields, T, sx) as a torch op whose backward is the adjoint kernel
    (jax.value_and_grad of loss_RPO, jax_scripts/adjoint_descent.py:91)."""
    dev = fields.device
    T = T if isinstance(T, torch.Tensor) else torch.tensor(float(T), dtype=torch.float64, device=dev)
    sx = sx if isinstance(sx, torch.Tensor) else torch.tensor(float(sx), dtype=torch.float64, device=dev)
    want = torch.is_grad_enabled() and any(t.requires_grad for t in (fields, T, sx))
    obj = Objective(param_dict, mode) if want else None
    return LossRPOFunction.apply(fields, T, sx, param_dict, mode, normalized, obj)
