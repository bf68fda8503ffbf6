"""FP64 CPU restatement of the reference hot path -- TEST INFRASTRUCTURE ONLY.

Every function follows one reference function line by line (file:line cited in
its docstring, paths relative to the mgolden30/ECS_MHD_2D project root).  The
functions are written once against a tiny array backend so that the same code
runs on numpy (forward map, CPU-baseline timing) and on torch-CPU (forward plus
``torch.func.jvp`` / ``torch.func.vjp``, which stand in for ``jax.jvp`` /
``jax.vjp``).  ``jax.lax.stop_gradient`` becomes ``Backend.stop_gradient``
(``detach`` on torch), ``lax.cond`` becomes a Python branch on primal values,
and ``jax.checkpoint`` (a memory optimisation that does not change values) is
dropped.
"""

from __future__ import annotations

import math

import numpy as np

try:  # torch is optional for the numpy-only users of this module
    import torch
except Exception:  # pragma: no cover
    torch = None

PI_LITERAL = 3.14159265358979323846  # mhd_jax.py:47 hard-codes pi


class Backend:
    """Minimal array API shared by the numpy and torch restatements."""

    def __init__(self, name):
        self.name = name
        self.is_torch = name == "torch"

    # --- creation -------------------------------------------------------
    def asarray(self, a, dtype=None):
        if self.is_torch:
            if isinstance(a, torch.Tensor):
                return a if dtype is None else a.to(dtype)
            return torch.as_tensor(np.asarray(a), dtype=dtype)
        return np.asarray(a, dtype=dtype)

    def real_dtype(self, bits=64):
        if self.is_torch:
            return torch.float64 if bits == 64 else torch.float32
        return np.float64 if bits == 64 else np.float32

    def arange(self, n, dtype):
        if self.is_torch:
            return torch.arange(n, dtype=dtype)
        return np.arange(n, dtype=dtype)

    def zeros(self, shape, dtype):
        if self.is_torch:
            return torch.zeros(shape, dtype=dtype)
        return np.zeros(shape, dtype=dtype)

    # --- math -----------------------------------------------------------
    def rfft2(self, a):
        return torch.fft.rfft2(a) if self.is_torch else np.fft.rfft2(a)

    def irfft2(self, a, n=None):
        if self.is_torch:
            return torch.fft.irfft2(a, s=None if n is None else (n, n))
        return np.fft.irfft2(a, s=None if n is None else (n, n))

    def exp(self, a):
        return torch.exp(a) if self.is_torch else np.exp(a)

    def conj(self, a):
        return torch.conj(a) if self.is_torch else np.conj(a)

    def flip(self, a, axis):
        return torch.flip(a, dims=(axis,)) if self.is_torch else np.flip(a, axis=axis)

    def roll(self, a, shift, axis):
        return torch.roll(a, shifts=shift, dims=axis) if self.is_torch else np.roll(a, shift, axis=axis)

    def mean(self, a):
        return torch.mean(a) if self.is_torch else np.mean(a)

    def maxabs(self, a):
        return torch.max(torch.abs(a)) if self.is_torch else np.max(np.abs(a))

    def isnan(self, a):
        return bool(torch.isnan(a)) if self.is_torch else bool(np.isnan(a))

    def stop_gradient(self, a):
        return a.detach() if self.is_torch else a

    def concatenate(self, arrs, axis):
        return torch.cat(arrs, dim=axis) if self.is_torch else np.concatenate(arrs, axis=axis)

    def expand_dims(self, a, axis):
        return torch.unsqueeze(a, axis) if self.is_torch else np.expand_dims(a, axis)

    def reshape(self, a, shape):
        return a.reshape(shape)

    def norm(self, a):
        return torch.linalg.norm(a) if self.is_torch else np.linalg.norm(a)


NUMPY = Backend("numpy")
TORCH = Backend("torch")


# ---------------------------------------------------------------------------
# mhd_jax.py
# ---------------------------------------------------------------------------

def construct_domain(n: int, xp: Backend = NUMPY, bits: int = 64):
    """Grid tables; restates ``construct_domain`` (jax_scripts/lib/mhd_jax.py:20-94).

    kx, ky, to_u, to_v are returned pre-masked (mhd_jax.py:87-90); the mask
    drops |k| >= n/3 and the mean mode (mhd_jax.py:65-70).
    """
    dt = xp.real_dtype(bits)
    grid = xp.arange(n, dt) / n * 2 * PI_LITERAL                  # :47
    if xp.is_torch:
        x, y = torch.meshgrid(grid, grid, indexing="ij")            # :52
    else:
        x, y = np.meshgrid(grid, grid, indexing="ij")
    k = np.fft.fftfreq(n, d=1.0 / n).astype(np.float64 if bits == 64 else np.float32)  # :55
    k = xp.asarray(k, dt)
    kx = xp.reshape(k, (-1, 1))                                      # :61
    ky = xp.reshape(k[: n // 2 + 1], (1, -1))                       # :62
    mask = (abs(kx) < n / 3) & (abs(ky) < n / 3)                     # :65
    mask = mask * (xp.asarray(np.ones((n, n // 2 + 1), bool)))
    if xp.is_torch:
        mask = mask.clone()
    mask[0, 0] = False                                               # :70
    k_sq = kx * kx + ky * ky                                         # :72
    k_sq[0, 0] = 1                                                   # :74
    inv_lap = -1 / k_sq                                              # :78
    inv_lap[0, 0] = 0
    inv_lap = inv_lap * mask
    to_u = ky / k_sq                                                 # :83
    to_v = -kx / k_sq
    kx = kx * mask                                                   # :87
    ky = ky * mask
    to_u = to_u * mask
    to_v = to_v * mask
    return {"x": x, "y": y, "kx": kx, "ky": ky, "mask": mask,
            "to_u": to_u, "to_v": to_v, "inv_lap": inv_lap}


def dissipation(param_dict, xp: Backend = NUMPY):
    """L = -(kx^2+ky^2)[nu, eta]; restates mhd_jax.py:97-102."""
    k_sq = param_dict["kx"] ** 2 + param_dict["ky"] ** 2
    coeffs = xp.asarray(np.array([param_dict["nu"], param_dict["eta"]], dtype=np.float64),
                        k_sq.dtype)
    coeffs = xp.reshape(coeffs, (2, 1, 1))
    return -k_sq * coeffs


def state_vel(fields, param_dict, include_dissipation, xp: Backend = NUMPY):
    """Nonlinear MHD time derivative; restates ``state_vel`` (mhd_jax.py:105-175)."""
    kx = param_dict["kx"]
    ky = param_dict["ky"]
    mask = param_dict["mask"]
    to_u = param_dict["to_u"]
    to_v = param_dict["to_v"]
    forcing = param_dict["forcing"]
    b0 = param_dict["b0"]
    fx = xp.irfft2(1j * kx * fields)                                 # :136
    fy = xp.irfft2(1j * ky * fields)                                 # :137
    fu = xp.irfft2(1j * to_u * fields)                               # :140
    fv = xp.irfft2(1j * to_v * fields)                               # :141
    bx = xp.reshape(xp.asarray(np.array([0.0, float(b0[0])]), fx.dtype), (2, 1, 1))  # :145
    by = xp.reshape(xp.asarray(np.array([0.0, float(b0[1])]), fx.dtype), (2, 1, 1))  # :146
    fu = fu + bx                                                     # :148
    fv = fv + by
    advection = fu * fx + fv * fy                                    # :152
    k_sq = (kx * kx + ky * ky) * mask                                # :154
    dwdt = -advection[..., 0, :, :] + advection[..., 1, :, :] + forcing   # :159
    dwdt = mask * xp.rfft2(dwdt)                                     # :160
    djdt = fu[..., 0, :, :] * fv[..., 1, :, :] - fv[..., 0, :, :] * fu[..., 1, :, :]  # :163
    djdt = k_sq * xp.rfft2(djdt)                                     # :164
    dwdt = xp.expand_dims(dwdt, -3)                                  # :167
    djdt = xp.expand_dims(djdt, -3)
    dfdt = xp.concatenate([dwdt, djdt], -3)                          # :169
    if include_dissipation:                                          # :171
        dfdt = dfdt + dissipation(param_dict, xp) * fields
    return dfdt


def state_vel_jvp(fields, tangent, param_dict, include_dissipation, xp: Backend = NUMPY):
    """Forward-mode derivative of ``state_vel`` (mhd_jax.py:105-175) at `fields`
    along `tangent` -- what ``jax.jvp(v_fn, (f,), (k,))`` evaluates inside tdrk4
    (timestepping.py:133).  The product rule applied to the statements of
    state_vel: the mean field b0 and the forcing are constants, every other
    factor is linear in the input."""
    kx = param_dict["kx"]
    ky = param_dict["ky"]
    mask = param_dict["mask"]
    to_u = param_dict["to_u"]
    to_v = param_dict["to_v"]
    b0 = param_dict["b0"]
    fx = xp.irfft2(1j * kx * fields)                                 # :136
    fy = xp.irfft2(1j * ky * fields)                                 # :137
    fu = xp.irfft2(1j * to_u * fields)                               # :140
    fv = xp.irfft2(1j * to_v * fields)                               # :141
    bx = xp.reshape(xp.asarray(np.array([0.0, float(b0[0])]), fx.dtype), (2, 1, 1))  # :145
    by = xp.reshape(xp.asarray(np.array([0.0, float(b0[1])]), fx.dtype), (2, 1, 1))  # :146
    fu = fu + bx                                                     # :148
    fv = fv + by
    dx = xp.irfft2(1j * kx * tangent)
    dy = xp.irfft2(1j * ky * tangent)
    du = xp.irfft2(1j * to_u * tangent)
    dv = xp.irfft2(1j * to_v * tangent)
    dadv = fu * dx + du * fx + fv * dy + dv * fy                     # d(:152)
    k_sq = (kx * kx + ky * ky) * mask                                # :154
    dwdt = -dadv[..., 0, :, :] + dadv[..., 1, :, :]                  # d(:159), forcing constant
    dwdt = mask * xp.rfft2(dwdt)                                     # :160
    djdt = (fu[..., 0, :, :] * dv[..., 1, :, :] + du[..., 0, :, :] * fv[..., 1, :, :]
            - fv[..., 0, :, :] * du[..., 1, :, :] - dv[..., 0, :, :] * fu[..., 1, :, :])  # d(:163)
    djdt = k_sq * xp.rfft2(djdt)                                     # :164
    dfdt = xp.concatenate([xp.expand_dims(dwdt, -3), xp.expand_dims(djdt, -3)], -3)
    if include_dissipation:                                          # :171
        dfdt = dfdt + dissipation(param_dict, xp) * tangent
    return dfdt


# ---------------------------------------------------------------------------
# timestepping.py
# ---------------------------------------------------------------------------

def rk4(f, t, steps, v_fn):
    """Classic RK4; restates timestepping.py:17-44."""
    h = t / steps
    for _ in range(steps):
        k1 = h * v_fn(f)
        k2 = h * v_fn(f + k1 / 2)
        k3 = h * v_fn(f + k2 / 2)
        k4 = h * v_fn(f + k3)
        f = f + k1 / 6 + k2 / 3 + k3 / 3 + k4 / 6
    return f


def lawson_rk4(f, t, steps, v_fn, L_diag, mask=None, xp: Backend = NUMPY):
    """Lawson integrating-factor RK4; restates timestepping.py:46-81 statement by statement."""
    h = t / steps                                                    # :69
    e = xp.exp(h / 2 * L_diag)                                       # :70
    if mask is not None:
        e = e * mask                                                 # :72
    for _ in range(steps):                                           # :81
        k1 = h * v_fn(f)                                             # :74
        f = e * f; k1 = e * k1                                       # :75
        k2 = h * v_fn(f + k1 / 2)                                    # :76
        k3 = h * v_fn(f + k2 / 2)                                    # :77
        f = e * f; k1 = e * k1; k2 = e * k2; k3 = e * k3             # :78
        k4 = h * v_fn(f + k3)                                        # :79
        f = f + k1 / 6 + k2 / 3 + k3 / 3 + k4 / 6                    # :80
    return f


def lawson_rk6(f, t, steps, v_fn, L_diag, mask=None, xp: Backend = NUMPY):
    """Lawson integrating-factor sixth-order RK; restates timestepping.py:83-125
    statement by statement (e = exp(h/6 L), applied after every stage)."""
    h = t / steps                                                    # :105
    e = xp.exp(h / 6 * L_diag)                                       # :106
    if mask is not None:
        e = e * mask                                                 # :108
    for _ in range(steps):                                           # :125
        k1 = h * v_fn(f)                                             # :110
        f = e * f; k1 = e * k1                                       # :111
        k2 = h * v_fn(f + k1 / 6)                                    # :112
        k3 = h * v_fn(f + k1 / 12 + k2 / 12)                         # :113
        f = e * f; k1 = e * k1; k2 = e * k2; k3 = e * k3             # :114
        k4 = h * v_fn(f - k2 * 4 / 33 + k3 * 5 / 11)                 # :115
        f = e * f; k1 = e * k1; k2 = e * k2; k3 = e * k3; k4 = e * k4   # :116
        k5 = h * v_fn(f - k1 / 4 - k2 * 29 / 44 + k3 * 31 / 22)      # :117
        f = e * f; k1 = e * k1; k2 = e * k2; k3 = e * k3; k4 = e * k4; k5 = e * k5   # :118
        k6 = h * v_fn(f + k1 * 3 / 11 + k2 * 8 / 33 - k3 * 4 / 11 + k4 / 11 + k5 * 14 / 33)   # :119
        f = e * f; k1 = e * k1; k2 = e * k2; k3 = e * k3; k4 = e * k4; k5 = e * k5; k6 = e * k6   # :120
        k7 = h * v_fn(f - k1 * 17 / 48 - k2 * 5 / 12 + k3 + k4 - k5 * 13 / 12 + k6 * 11 / 16)   # :121
        f = e * f; k1 = e * k1; k2 = e * k2; k3 = e * k3; k4 = e * k4; k5 = e * k5; k6 = e * k6; k7 = e * k7  # :122
        k8 = h * v_fn(f + k1 * 20 / 39 + k2 * 12 / 39 - k3 * 31 / 39 - k4 / 39 + k5 * 34 / 39
                      - k6 * 11 / 39 + k7 * 16 / 39)                 # :123
        f = f + 13 / 200 * (k1 + k8) + 4 / 25 * (k3 + k7) + 11 / 40 * (k4 + k6)   # :124
    return f


def tdrk4(f, t, steps, v_fn, jac_fn):
    """Two-derivative RK4; restates timestepping.py:127-149.  jac_fn(f, k) is the
    Jacobian-vector product of v_fn at f along k (jax.jvp at :133)."""
    h = t / steps                                                    # :132
    for _ in range(steps):                                           # :148
        k1 = h * v_fn(f)                                             # :137
        a1 = h * jac_fn(f, k1)                                       # :138
        f_temp = f + k1 / 2 + a1 / 8                                 # :140
        k2 = h * v_fn(f_temp)                                        # :141
        a2 = h * jac_fn(f_temp, k2)                                  # :142
        f = f + k1 + a1 / 6 + a2 / 3                                 # :144
    return f


def lawson_rk43(x, vel_fn, diag_L, t, h=1e-2, atol=1e-4, max_steps_per_checkpoint=1024,
                checkpoints=1, xp: Backend = NUMPY, n=None):
    """Adaptive Lawson-RK4(3); restates ``lawson_rk43`` (timestepping.py:151-335).

    Reproduces the reference's quirks: the exponential ``e`` is not masked
    (:263); on rejection the carried k1 keeps both twiddles, k1 <- e^2 k1
    (:267,:275,:297); h is a stop-gradient constant (:308); completed
    iterations are no-ops within a fixed trip count (:313-321).
    ``n`` is the grid side, used for the real-space error norm (:290).
    Returns (x, info) with info = completed, s, accepted, rejected, fevals,
    hs, and ``acc_seq`` (one bool per attempted step, in order).
    """
    total = max_steps_per_checkpoint * checkpoints
    hs = np.zeros(total)                                             # :239
    mod_L = t * diag_L                                               # :242
    mod_vel_fn = lambda z: t * vel_fn(z)                             # :243
    s = 0.0
    k1 = mod_vel_fn(x)                                               # :255
    fevals, accepted, rejected = 1, 0, 0
    acc_seq = []
    complete_fn = lambda s_: abs(s_ - 1.0) < 1e-10                   # :313
    for _ in range(total):
        if complete_fn(s):                                           # :317
            continue
        x0 = x
        e = xp.exp(mod_L * h / 2)                                    # :263
        x = e * x0                                                   # :266
        k1 = e * k1                                                  # :267
        k2 = mod_vel_fn(x + h * k1 / 2)                              # :270
        k3 = mod_vel_fn(x + h * k2 / 2)                              # :271
        x = e * x; k1 = e * k1; k2 = e * k2; k3 = e * k3             # :274-277
        k4 = mod_vel_fn(x + h * k3)                                  # :280
        xf = x + h * (k1 / 6 + k2 / 3 + k3 / 3 + k4 / 6)             # :281
        k5 = mod_vel_fn(xf)                                          # :282
        fevals += 4                                                  # :285
        err = h * (k5 - k4) / 6                                      # :288
        err = xp.irfft2(err, n)                                      # :290
        err = float(xp.maxabs(xp.stop_gradient(err)))                # :291
        hs[accepted + rejected] = h                                  # :294
        if err < atol:                                               # :297
            x, k1, s, accepted = xf, k5, s + h, accepted + 1
            acc_seq.append(True)
        else:
            x, rejected = x0, rejected + 1
            acc_seq.append(False)
        if math.isnan(err):                                          # :300-302
            h = h / 2
        else:
            h = h * 0.9 * (atol / err) ** (1 / 4) if err != 0 else float("inf")
        overshoot = s + h - 1                                        # :304-307
        h = h - max(overshoot, 0.0)
        h = float(h)                                                 # :308 stop_gradient
    info = {"completed": complete_fn(s), "s": s, "accepted": accepted,
            "rejected": rejected, "fevals": fevals, "hs": hs, "acc_seq": acc_seq}
    return x, info


# ---------------------------------------------------------------------------
# symmetry.py
# ---------------------------------------------------------------------------

def shift_x(f, s, param_dict, xp: Backend = NUMPY):
    """exp(i kx s) f with masked kx; restates symmetry.py:4-5."""
    return xp.exp(1j * param_dict["kx"] * s) * f


def shift_reflect(f, n, param_dict, xp: Backend = NUMPY):
    """Shift y by n*2pi/8 and reflect x for odd n; restates symmetry.py:7-19."""
    n = int(n)
    s = (n * 2 * math.pi) / 8                                        # :11 (jnp.pi in x64)
    f = xp.exp(1j * param_dict["ky"] * s) * f                        # :12
    if n % 2 == 1:
        f = xp.flip(f, -2)                                           # :15
        f = xp.roll(f, 1, -2)                                        # :16
        f = -f                                                       # :18
    return f


def rot180(f, xp: Backend = NUMPY):
    """conj(f) with channel signs [1,-1]; restates symmetry.py:21-25."""
    f = xp.conj(f)
    sign = xp.reshape(xp.asarray(np.array([1.0, -1.0]), f.real.dtype), (2, 1, 1))
    return sign * f


# ---------------------------------------------------------------------------
# loss_functions.py
# ---------------------------------------------------------------------------

def mismatch_RPO(input_dict, param_dict, mode, xp: Backend = NUMPY):
    """Restates ``mismatch_RPO`` (loss_functions.py:9-96) for all five modes
    (RK4, Lawson_RK4, Lawson_RK6, Lawson_RK43, TDRK4).  Returns (f0, f, info)."""
    f0 = input_dict["fields"]
    T = input_dict["T"]
    sx = input_dict["sx"]
    n = f0.shape[-1]
    f0 = xp.rfft2(f0)                                                # :45
    if mode == "RK4":                                                # :49-56
        nc, ms = int(param_dict["num_checkpoints"]), int(param_dict["ministeps"])
        v_fn = lambda f: state_vel(f, param_dict, True, xp)
        f = f0
        for _ in range(nc):
            f = rk4(f, T / nc, ms, v_fn)
        info = None
    elif mode == "Lawson_RK4":                                       # :57-65
        nc, ms = int(param_dict["num_checkpoints"]), int(param_dict["ministeps"])
        v_fn = lambda f: state_vel(f, param_dict, False, xp)
        L_diag = dissipation(param_dict, xp)
        f = f0
        for _ in range(nc):
            f = lawson_rk4(f, T / nc, ms, v_fn, L_diag, mask=param_dict["mask"], xp=xp)
        info = None
    elif mode == "Lawson_RK6":                                       # :66-71
        v_fn = lambda f: state_vel(f, param_dict, False, xp)
        L_diag = dissipation(param_dict, xp)
        f = lawson_rk6(f0, T, int(param_dict["steps"]), v_fn, L_diag, mask=param_dict["mask"], xp=xp)
        info = None
    elif mode == "TDRK4":                                            # :78-85
        nc, ms = int(param_dict["num_checkpoints"]), int(param_dict["ministeps"])
        v_fn = lambda f: state_vel(f, param_dict, True, xp)
        if xp is TORCH:   # jax.jvp of v_fn (timestepping.py:133)
            jac_fn = lambda f, k: torch.func.jvp(v_fn, (f,), (k,))[1]
        else:             # the same derivative written out (product rule of state_vel)
            jac_fn = lambda f, k: state_vel_jvp(f, k, param_dict, True, xp)
        f = f0
        for _ in range(nc):
            f = tdrk4(f, T / nc, ms, v_fn, jac_fn)
        info = None
    elif mode == "Lawson_RK43":                                      # :72-77
        vel_fn = lambda f: state_vel(f, param_dict, False, xp)
        L_diag = dissipation(param_dict, xp)
        ad = param_dict["adaptive_dict"]
        f, info = lawson_rk43(f0, vel_fn, L_diag, T, h=1e-2, atol=ad["atol"],
                              max_steps_per_checkpoint=ad["max_steps_per_checkpoint"],
                              checkpoints=ad["checkpoints"], xp=xp, n=n)
    else:                                                            # :86-88
        raise ValueError(f"You selected mode = {mode}, which does not exist.")
    f = shift_x(f, sx, param_dict, xp)                               # :91
    f = shift_reflect(f, param_dict["shift_reflect_ny"], param_dict, xp)  # :92
    if param_dict["rot"]:                                            # :93
        f = rot180(f, xp)
    return f0, f, info


def loss_RPO(input_dict, param_dict, mode, xp: Backend = NUMPY):
    """mean(irfft2(f - f0)^2); restates loss_functions.py:99-111."""
    f0, f, info = mismatch_RPO(input_dict, param_dict, mode, xp)
    n = input_dict["fields"].shape[-1]
    diff = xp.irfft2(f - f0, n)
    return xp.mean(diff * diff), info


def phase_conditions(f0, param_dict, xp: Backend = NUMPY, n=None):
    """Phase conditions with value 0; restates loss_functions.py:113-130."""
    vt = state_vel(f0, param_dict, True, xp)
    vx = 1j * param_dict["kx"] * f0
    vt = xp.stop_gradient(xp.irfft2(vt, n))
    vx = xp.stop_gradient(xp.irfft2(vx, n))
    f0 = xp.irfft2(f0, n)
    pt = xp.mean(vt * f0)
    px = xp.mean(vx * f0)
    pt = pt - xp.stop_gradient(pt)
    px = px - xp.stop_gradient(px)
    return pt, px


def objective_RPO(input_dict, param_dict, mode, xp: Backend = NUMPY):
    """{"fields": irfft2(f0 - f), "T": pt, "sx": px}; restates loss_functions.py:132-148."""
    f0, f, info = mismatch_RPO(input_dict, param_dict, mode, xp)
    n = input_dict["fields"].shape[-1]
    pt, px = phase_conditions(f0, param_dict, xp, n)
    return {"fields": xp.irfft2(f0 - f, n), "T": pt, "sx": px}


# ---------------------------------------------------------------------------
# param dict helpers (dictionaryIO.recompute_grid_information, dictionaryIO.py:64-78)
# ---------------------------------------------------------------------------

def make_param_dict(n, nu, eta, b0=(0.0, 0.1), forcing="kolmogorov", xp: Backend = NUMPY,
                    bits=64, **extra):
    """Grid + physics parameters.  ``forcing`` is "kolmogorov" (-4cos(4y), the
    fixtures' ``forcing_str``), "kolmogorov+" (+4cos(4y), the synthetic
    workloads' text), a callable f(x, y) or an [n, n] array."""
    pd = construct_domain(n, xp, bits)
    x, y = pd["x"], pd["y"]
    if isinstance(forcing, str):
        amp = {"kolmogorov": -4.0, "kolmogorov+": 4.0}[forcing]
        fr = amp * (torch.cos(4 * y) if xp.is_torch else np.cos(4 * y))
    elif callable(forcing):
        fr = forcing(x, y)
    else:
        fr = xp.asarray(forcing, x.dtype)
    pd.update({"nu": float(nu), "eta": float(eta), "b0": [float(b0[0]), float(b0[1])],
               "forcing": fr})
    pd.update(extra)
    return pd


def change_resolution(f, n):
    """Restates change_resolution (jax_scripts/upscale_state.py:29-47) in numpy."""
    m = f.shape[-1]
    F = np.fft.fft2(f)
    F2 = np.zeros(f.shape[:-2] + (n, n), dtype=np.complex128)
    m2 = min(m, n) // 2                                              # :36
    F2[..., 0:m2, 0:m2] = F[..., 0:m2, 0:m2]                         # :40-43
    F2[..., n - m2:, 0:m2] = F[..., -m2:, 0:m2]
    F2[..., 0:m2, n - m2:] = F[..., 0:m2, -m2:]
    F2[..., n - m2:, n - m2:] = F[..., -m2:, -m2:]
    return np.real(np.fft.ifft2(F2) * (n / m) ** 2)                  # :45, :47


def compute_observables(f, param_dict):
    """Restates compute_observables (jax_scripts/projection.py:19-46) in numpy."""
    n = f.shape[-2]
    u = np.fft.irfft2(1j * param_dict["to_u"] * f[0], s=(n, n))                # :32
    v = np.fft.irfft2(1j * param_dict["to_v"] * f[0], s=(n, n))                # :33
    force = np.fft.rfft2(param_dict["forcing"])                                 # :35
    fx = np.fft.irfft2(1j * param_dict["to_u"] * force, s=(n, n))               # :36
    fy = np.fft.irfft2(1j * param_dict["to_v"] * force, s=(n, n))               # :37
    injection = np.mean(u * fx + v * fy)                                        # :40
    d = np.mean(np.square(np.fft.irfft2(f, s=(n, n))), axis=(-1, -2))           # :43
    return np.array([injection, param_dict["nu"] * d[0] + param_dict["eta"] * d[1]])   # :44-45


def laminar_flow(param_dict):
    """Restates laminar_flow (jax_scripts/projection.py:49-73)."""
    alpha = param_dict["b0"][1]
    L = np.sqrt(param_dict["eta"] * param_dict["nu"]) / alpha
    k = 4.0
    y = param_dict["y"]
    U0 = param_dict["eta"] / (alpha * alpha * (1 + L * L * k * k))
    B0 = 1.0 / (k * alpha * (1 + L * L * k * k))
    return np.stack([-U0 * k * np.cos(k * y), B0 * k * np.sin(k * y)])


def ravel_dict(d, xp: Backend = NUMPY):
    """Flatten {"T","fields","sx"} in jax ravel_pytree order (sorted keys): [T, fields, sx]."""
    if xp.is_torch:
        return torch.cat([d["T"].reshape(1), d["fields"].reshape(-1), d["sx"].reshape(1)])
    return np.concatenate([np.reshape(d["T"], 1), np.reshape(d["fields"], -1), np.reshape(d["sx"], 1)])


def unravel_dict(v, n):
    return {"T": v[0], "fields": v[1:-1].reshape(2, n, n), "sx": v[-1]}


# ---------------------------------------------------------------------------
# linalg.py / utils.py
# ---------------------------------------------------------------------------

def gmres(A, b, inner, outer=1, preconditioner_list=()):
    """MGS-Arnoldi GMRES without restarts; restates linalg.py:12-98 (numpy)."""
    n = b.size
    Q = np.zeros((n, inner + 1))
    H = np.zeros((inner + 1, inner))

    def precond(v):
        for M in preconditioner_list:
            v = M(v)
        return v

    b = precond(b)
    Q[:, 0] = b / np.linalg.norm(b)
    for k in range(inner):
        Aq = precond(A(Q[:, k]))
        for j in range(k + 1):
            hj = np.dot(Aq, Q[:, j])
            Aq = Aq - hj * Q[:, j]
            H[j, k] = hj
        hk1 = np.linalg.norm(Aq)
        H[k + 1, k] = hk1
        Q[:, k + 1] = Aq / hk1
    b2 = Q.T @ b
    y = np.linalg.lstsq(H, b2, rcond=None)[0]
    x = Q[:, :inner] @ y
    rel_res = np.linalg.norm(precond(A(x)) - b) / np.linalg.norm(b)
    return x, rel_res


def line_search_unravel(x, step, obj, unravel_fn, f_vec, flatten, max_iters=20):
    """Damped step that must decrease |f|; restates utils.py:17-58."""
    norm_orig = np.linalg.norm(f_vec)
    damp, done = 1.0, False
    for _ in range(max_iters):
        if done:
            continue
        x_temp = x - damp * step
        norm_temp = np.linalg.norm(flatten(obj(unravel_fn(x_temp))))
        improved = norm_temp < norm_orig
        if improved:
            x = x_temp
        else:
            damp = damp / 2.0
        done = done or improved
    return x, damp
