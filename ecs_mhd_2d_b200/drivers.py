"""Newton-GMRES and adjoint-descent iterations on top of the device path
(reference drivers: jax_scripts/newton.py:151-215, jax_scripts/adjoint_descent.py:93-114).
"""

from __future__ import annotations

import torch

from .autodiff import Objective, loss_and_grad, vjp
from .linalg import block_gmres, gmres, newton_gmres_hookstep_v2
from .loss_functions import dealias
from .utils import flatten, line_search_unravel, relative_error_RPO, unflatten


def _as_device_dict(d, device="cuda"):
    f = d["fields"] if isinstance(d["fields"], torch.Tensor) else torch.as_tensor(d["fields"])
    return {"fields": f.to(device=device, dtype=torch.float64).contiguous(),
            "T": float(d["T"]), "sx": float(d["sx"])}


def newton_gmres_update(input_dict, param_dict, mode, inner=16, use_transpose=True, do_line_search=True,
                        default_damp=0.1, jac_obj=None):
    """One Newton-GMRES update (newton.py:151-215).  Solves J s = f (or
    J^T J s = J^T f with use_transpose) with `inner` Krylov vectors, applies a
    line search, and dealiases.  `jac_obj` (optional) is a second Objective
    used for the Jacobian products, e.g. an FP32 one for mixed precision.
    Returns (new_input_dict, stats)."""
    obj = Objective(param_dict, mode)
    jac = jac_obj or obj
    x_dict = _as_device_dict(input_dict)
    n = x_dict["fields"].shape[-1]
    f = obj(x_dict)
    b = flatten(f)

    def cast_in(d):
        if jac is obj:
            return d
        dt = jac.param_dict["x"].dtype
        return {"fields": d["fields"].to(dt), "T": d["T"], "sx": d["sx"]}

    def A(v):
        t = unflatten(v, n)
        out = jac.jvp(cast_in(x_dict), cast_in({"fields": t["fields"], "T": t["T"], "sx": t["sx"]}))
        return flatten({"fields": out["fields"].to(torch.float64), "T": out["T"], "sx": out["sx"]})

    precond = []
    if use_transpose:
        _, jacT = vjp(jac, cast_in(x_dict))

        def A_T(v):
            t = unflatten(v, n)
            g = jacT({"fields": t["fields"].to(jac.param_dict["x"].dtype).contiguous(), "T": t["T"], "sx": t["sx"]})[0]
            return flatten({"fields": g["fields"].to(torch.float64), "T": g["T"], "sx": g["sx"]})

        precond = [A_T]
    step, gmres_res = gmres(A, b, inner, 1, precond)
    x = flatten(x_dict)
    unravel = lambda v: unflatten(v, n)
    if do_line_search:
        x, damp = line_search_unravel(x, step, obj, unravel, b, max_iters=20)
    else:
        damp = default_damp
        x = x - damp * step
    new = unravel(x)
    rel_err = relative_error_RPO(x_dict, f)
    new = {"fields": dealias(new["fields"].contiguous(), param_dict), "T": float(new["T"]), "sx": float(new["sx"])}
    stats = {"rel_err": float(rel_err), "|f|": float(torch.linalg.norm(b)), "gmres_rel_res": float(gmres_res),
             "damp": damp, "T": new["T"], "sx": new["sx"]}
    return new, stats


def newton_hookstep_iteration(input_dict, param_dict, mode, inner=64, s=100.0, obj=None):
    """One iteration of the trust-region Newton driver
    (jax_scripts/newton_hookstep_v2.py:95-121): objective, Krylov space of the
    JVP at the current point, newton_gmres_hookstep_v2 with step bound s, then
    dealias.  Returns (new_input_dict, s, stats) with the driver's printed
    quantities (rel_err, |f|, rel_res, T, sx)."""
    obj = obj or Objective(param_dict, mode)
    x_dict = _as_device_dict(input_dict)
    n = x_dict["fields"].shape[-1]
    f = obj(x_dict)
    f_vec = flatten(f)

    def A(v):
        t = unflatten(v, n)
        return flatten(obj.jvp(x_dict, {"fields": t["fields"].contiguous(), "T": t["T"], "sx": t["sx"]}))

    new, s, rel_res = newton_gmres_hookstep_v2(A, f_vec, inner, s, obj, x_dict)   # newton_hookstep_v2.py:108
    rel_err = relative_error_RPO(new, f)                          # :112, |f| over the updated fields
    new = {"fields": dealias(new["fields"].contiguous(), param_dict), "T": float(new["T"]),
           "sx": float(new["sx"])}                                 # :116-119
    stats = {"rel_err": float(rel_err), "|f|": float(torch.linalg.norm(f_vec)), "rel_res": float(rel_res),
             "s": s, "T": new["T"], "sx": new["sx"]}
    return new, s, stats


def newton_block_gmres_update(input_dict, param_dict, mode, block=8, m=4, seed=0, do_line_search=True, obj=None):
    """Newton update whose linear solve is block_gmres (jax_scripts/lib/
    linalg.py:340-427) over {B, JB, ..., J^m B}: B holds the residual and
    block-1 seeded random directions, and every application of J is ONE
    batched JVP of `block` tangents, where sequential GMRES issues one tangent
    per Krylov vector.  Line search and dealiasing as in newton_gmres_update.
    Returns (new_input_dict, stats)."""
    import numpy as np
    obj = obj or Objective(param_dict, mode)
    x_dict = _as_device_dict(input_dict)
    n = x_dict["fields"].shape[-1]
    f = obj(x_dict)
    b = flatten(f)
    nv = b.numel()
    R = torch.as_tensor(np.random.default_rng(seed).standard_normal((nv, block - 1)), device=b.device)
    B0 = torch.cat([b.reshape(nv, 1), R], dim=1)

    def A(Bk):
        s_ = Bk.shape[1]
        t = Bk.t().contiguous()
        out = obj.jvp(x_dict, {"fields": t[:, 1:-1].reshape(s_, 2, n, n).contiguous(), "T": t[:, 0].contiguous(),
                               "sx": t[:, -1].contiguous()})
        return torch.cat([out["T"].reshape(1, s_), out["fields"].reshape(s_, -1).t(), out["sx"].reshape(1, s_)], 0)

    step = block_gmres(A, b, m, B0)
    res = float(torch.linalg.norm(A(step.reshape(nv, 1)).reshape(-1) - b) / torch.linalg.norm(b))
    x = flatten(x_dict)
    unravel = lambda v: unflatten(v, n)
    if do_line_search:
        x, damp = line_search_unravel(x, step, obj, unravel, b, max_iters=20)
    else:
        damp = 1.0
        x = x - step
    new = unravel(x)
    rel_err = relative_error_RPO(x_dict, f)
    new = {"fields": dealias(new["fields"].contiguous(), param_dict), "T": float(new["T"]), "sx": float(new["sx"])}
    return new, {"rel_err": float(rel_err), "|f|": float(torch.linalg.norm(b)), "block_gmres_rel_res": res,
                 "damp": damp, "T": new["T"], "sx": new["sx"]}


def second_directional_derivative(obj, input_dict, v, eps=None):
    """K(v) = d^2 objective[v, v] at input_dict for a flat direction v ([T,
    fields, sx]), as the nested jax.jvp of jax_scripts/acceleration.py:127-129
    computes it.  Here it is the central difference of two JVPs along v at
    x +- eps v (each a linearisation and one tangent on the device), error
    O(eps^2) (a few 1e-7 relative at the default eps = 1e-5 max(|x|, 1) / |v|),
    except for the two phase conditions: they are linear in the state with
    stop-gradient coefficients (loss_functions.py:113-130), so their second
    derivative is exactly zero, while the difference would also differentiate
    those coefficients; their entries are set to zero.  `obj` should be an
    Objective of its own (its linearisations move to x +- eps v)."""
    x_dict = _as_device_dict(input_dict)
    n = x_dict["fields"].shape[-1]
    x = flatten(x_dict)
    v = v.to(torch.float64)
    if eps is None:
        eps = 1e-5 * max(float(torch.linalg.norm(x)), 1.0) / float(torch.linalg.norm(v))
    t = unflatten(v, n)
    tan = {"fields": t["fields"].contiguous(), "T": t["T"], "sx": t["sx"]}

    def jv(xs):
        d = unflatten(xs, n)
        return flatten(obj.jvp({"fields": d["fields"].contiguous(), "T": float(d["T"]), "sx": float(d["sx"])}, tan))

    k = (jv(x + eps * v) - jv(x - eps * v)) / (2 * eps)
    k[0] = 0.0    # pt (flat order [pt, fields, px])
    k[-1] = 0.0   # px
    return k


def geodesic_acceleration_update(input_dict, param_dict, mode, inner=16, obj=None, obj_k=None):
    """One Newton-GMRES update with geodesic acceleration
    (jax_scripts/acceleration.py:103-168): step1 solves J s = -f, step2 solves
    J s = -K(step1)/2 with the second directional derivative K, both by GMRES
    with the transpose preconditioner; x <- x + step1 + step2, then dealias.
    K is the central difference of two JVPs (second_directional_derivative)
    where the reference nests jax.jvp.  Returns (new_input_dict, stats)."""
    obj = obj or Objective(param_dict, mode)
    obj_k = obj_k or Objective(param_dict, mode)
    x_dict = _as_device_dict(input_dict)
    n = x_dict["fields"].shape[-1]
    f = obj(x_dict)
    b = -flatten(f)                                                    # acceleration.py:114

    def J(v):                                                          # :117
        t = unflatten(v, n)
        return flatten(obj.jvp(x_dict, {"fields": t["fields"].contiguous(), "T": t["T"], "sx": t["sx"]}))

    _, jacT = vjp(obj, x_dict)                                         # :120-121

    def J_T(v):
        t = unflatten(v, n)
        g = jacT({"fields": t["fields"].contiguous(), "T": t["T"], "sx": t["sx"]})[0]
        return flatten({"fields": g["fields"], "T": g["T"], "sx": g["sx"]})

    step1, res1 = gmres(J, b, inner, 1, [J_T])                         # :124
    r = -second_directional_derivative(obj_k, x_dict, step1) / 2       # :127-131
    step2, res2 = gmres(J, r, inner, 1, [J_T])                         # :134
    new = unflatten(flatten(x_dict) + step1 + step2, n)                # :137-142
    rel_err = relative_error_RPO(new, f)                               # :148
    new = {"fields": dealias(new["fields"].contiguous(), param_dict), "T": float(new["T"]),
           "sx": float(new["sx"])}                                     # :163-167
    stats = {"rel_err": float(rel_err), "|f|": float(torch.linalg.norm(b)), "gmres_rel_res": float(res1),
             "gmres_rel_res_2": float(res2), "|step1|": float(torch.linalg.norm(step1)),
             "|step2|": float(torch.linalg.norm(step2)), "T": new["T"], "sx": new["sx"]}
    return new, stats


def init_adam(params):
    """Zero moments (jax_scripts/lib/adam.py:7-20)."""
    return ({k: 0 * torch.as_tensor(v) for k, v in params.items()},
            {k: 0 * torch.as_tensor(v) for k, v in params.items()})


def adam_update(params, grads, m, v, t, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
    """One ADAM step on dicts (jax_scripts/lib/adam.py:23-61)."""
    m = {k: beta1 * m[k] + (1 - beta1) * grads[k] for k in params}
    v = {k: beta2 * v[k] + (1 - beta2) * grads[k] ** 2 for k in params}
    m_hat = {k: m[k] / (1 - beta1 ** t) for k in params}
    v_hat = {k: v[k] / (1 - beta2 ** t) for k in params}
    params = {k: params[k] - lr * m_hat[k] / (torch.sqrt(v_hat[k]) + eps) for k in params}
    return params, m, v


def adjoint_descent_step(input_dict, param_dict, mode, m, v, t, lr=1e-2):
    """One adjoint-descent iteration (adjoint_descent.py:93-114): gradient of
    loss_RPO by the adjoint kernels, ADAM update, dealias.  Returns
    (new_input_dict, m, v, loss, info)."""
    x = _as_device_dict(input_dict)
    (loss, info), g = loss_and_grad(x, param_dict, mode)
    params = {"fields": x["fields"], "T": torch.tensor(x["T"], dtype=torch.float64, device="cuda"),
              "sx": torch.tensor(x["sx"], dtype=torch.float64, device="cuda")}
    grads = {"fields": g["fields"], "T": g["T"].reshape(()), "sx": g["sx"].reshape(())}
    if t == 1 and not m:
        m, v = init_adam(params)
    params, m, v = adam_update(params, grads, m, v, t, lr=lr, beta1=0.9, beta2=0.999, eps=1e-6)
    new = {"fields": dealias(params["fields"].contiguous(), param_dict), "T": float(params["T"]),
           "sx": float(params["sx"])}
    return new, m, v, float(loss), info


def mixed_precision_objectives(param_dict, mode):
    """(FP64 objective for residuals, FP32 objective for Jacobian products) over
    the same physics: time stepping and JVP/VJP in FP32, the Newton residual,
    Arnoldi and Hessenberg solve in FP64."""
    from .mhd import make_param_dict
    n = param_dict["x"].shape[-1]
    keep = {k: v for k, v in param_dict.items() if k not in ("x", "y", "kx", "ky", "mask", "to_u", "to_v",
                                                             "inv_lap", "forcing", "nu", "eta", "b0")}
    f64 = param_dict["forcing"].detach().to("cpu", torch.float64).numpy()
    pd32 = make_param_dict(n, param_dict["nu"], param_dict["eta"], b0=param_dict["b0"], forcing=f64,
                           data_type=torch.float32, **keep)
    return Objective(param_dict, mode), Objective(pd32, mode)


def mixed_precision_newton(input_dict, param_dict, mode, iters=3, inner=16, use_transpose=True, refine=0):
    """Inexact Newton with FP32 Jacobian products (stepping, JVP, VJP in FP32) and
    FP64 residuals, Arnoldi and least squares, followed by `refine` Newton steps
    with FP64 Jacobian products.  `use_transpose` selects the Gauss-Newton form
    J^T J s = J^T f as jax_scripts/newton.py:151-187 does by default.  The FP32
    products perturb each GMRES solve by about the FP32 rounding of the
    linearised flow, far below the inexactness of a 16-vector Krylov solve, so
    the iteration follows the FP64 one step for step.  Returns (state,
    history); history[-1] holds the final FP64 relative residual."""
    _, obj32 = mixed_precision_objectives(param_dict, mode)
    x = input_dict
    hist = []
    for _ in range(iters):
        x, st = newton_gmres_update(x, param_dict, mode, inner=inner, use_transpose=use_transpose, jac_obj=obj32)
        st["jacobian"] = "fp32"
        hist.append(st)
    for _ in range(refine):
        x, st = newton_gmres_update(x, param_dict, mode, inner=inner, use_transpose=True)
        st["jacobian"] = "fp64"
        hist.append(st)
    f = Objective(param_dict, mode)(_as_device_dict(x))
    hist.append({"final_rel_err": float(relative_error_RPO(_as_device_dict(x), f))})
    return x, hist


def floquet_operator(input_dict, param_dict, mode="TDRK4", obj=None):
    """J_fl(tangents): the Jacobian of the masked, symmetry-shifted flow map
    f0 -> irfft2(mask . mismatch_RPO(f0)) that jax_scripts/floquet.py:40-56
    differentiates (jax.jvp, vmapped over a block of tangents), at fixed T and sx.
    objective_RPO's fields output is irfft2(f0 - g Phi_T(f0)), so the map's
    derivative is dealias(t - d_objective(t)): one batched ecs_jvp per call.
    Returns a function of tangents [B, 2, n, n] (device, FP64)."""
    obj = obj or Objective(param_dict, mode)
    x = _as_device_dict(input_dict)

    def apply(tang):
        B = tang.shape[0]
        zero = torch.zeros(B, dtype=torch.float64)
        d = obj.jvp(x, {"fields": tang.contiguous(), "T": zero, "sx": zero})
        return dealias((tang - d["fields"]).contiguous(), param_dict)
    return apply


def floquet_power_iteration(input_dict, param_dict, mode="TDRK4", block_size=32, maxit=256, seed=0,
                            tangents=None):
    """Block power iteration for the leading Floquet multipliers of an RPO
    (jax_scripts/floquet.py:58-99): `maxit` applications of J_fl to a block of
    `block_size` tangents, each followed by a reduced QR re-orthonormalisation,
    then R = Q J_fl(Q)^T (Schur factor estimate).  Seeded normal start vectors
    (numpy PCG64 here; the reference uses jax.random).  Returns (R, Q) with Q
    [block_size, 2, n, n]."""
    import numpy as np
    apply = floquet_operator(input_dict, param_dict, mode)
    n = _as_device_dict(input_dict)["fields"].shape[-1]
    if tangents is None:
        tangents = torch.as_tensor(np.random.default_rng(seed).standard_normal((block_size, 2, n, n)), device="cuda")
    q = tangents.to(device="cuda", dtype=torch.float64)
    B = q.shape[0]

    def orth(t):
        Qm, _ = torch.linalg.qr(t.reshape(B, -1).T, mode="reduced")   # floquet.py:90-92
        return Qm.T.reshape(B, 2, n, n).contiguous()

    for _ in range(maxit):
        q = orth(apply(q))
    R = q.reshape(B, -1) @ apply(q).reshape(B, -1).T                     # floquet.py:95-98
    return R, q
