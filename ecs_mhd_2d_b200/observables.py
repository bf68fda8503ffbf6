"""Energy observables along an orbit (reference: jax_scripts/projection.py).

For each state the energy injection by the forcing and the dissipation rate,
along the orbit of a solution (TDRK4 steps of T/steps, the reference script's
integrator), normalised by their values for the laminar flow.  The stepping is
`timestepping.integrate` on the device; the observables are a few FFTs of one
state, evaluated with torch on the state's device.
"""

from __future__ import annotations

import torch

from .timestepping import integrate


def compute_observables(f, param_dict):
    """[injection, dissipation] of an rfft2 state f [2, n, n//2+1]
    (projection.py:19-46): injection = mean(u fx + v fy) with (u, v) the
    velocity of f[0] and (fx, fy) that of the forcing's curl-free part as the
    reference computes it; dissipation = nu mean(w^2) + eta mean(j^2)."""
    n = f.shape[-2]
    to_u = param_dict["to_u"].to(f.device)
    to_v = param_dict["to_v"].to(f.device)
    u = torch.fft.irfft2(1j * to_u * f[0], s=(n, n))
    v = torch.fft.irfft2(1j * to_v * f[0], s=(n, n))
    force = torch.fft.rfft2(param_dict["forcing"].to(device=f.device, dtype=u.dtype))
    fx = torch.fft.irfft2(1j * to_u * force, s=(n, n))
    fy = torch.fft.irfft2(1j * to_v * force, s=(n, n))
    injection = torch.mean(u * fx + v * fy)
    sq = torch.mean(torch.square(torch.fft.irfft2(f, s=(n, n))), dim=(-1, -2))
    dissipation = param_dict["nu"] * sq[0] + param_dict["eta"] * sq[1]
    return torch.stack([injection, dissipation])


def laminar_flow(param_dict):
    """The laminar state [2, n, n] of the reference (projection.py:49-73):
    w = -U0 k cos(k y), j = B0 k sin(k y), k = 4, with L = sqrt(eta nu)/alpha,
    alpha = b0[1], U0 = eta / (alpha^2 (1 + L^2 k^2)), B0 = 1 / (k alpha (1 + L^2 k^2))."""
    alpha = float(param_dict["b0"][1])
    nu, eta = float(param_dict["nu"]), float(param_dict["eta"])
    L = (eta * nu) ** 0.5 / alpha
    k = 4.0
    y = param_dict["y"]
    U0 = eta / (alpha * alpha * (1 + L * L * k * k))
    B0 = 1.0 / (k * alpha * (1 + L * L * k * k))
    return torch.stack([-U0 * k * torch.cos(k * y), B0 * k * torch.sin(k * y)])


def projection(input_dict, param_dict, steps=None, device="cuda"):
    """Observables [2, steps] along the orbit of input_dict (projection.py:80-116):
    step i holds compute_observables of the state after i TDRK4 steps of
    dt = T / steps (steps = param_dict["steps"] by default), divided by those
    of the laminar flow."""
    steps = int(steps if steps is not None else param_dict["steps"])
    fields = torch.as_tensor(input_dict["fields"], dtype=torch.float64, device=device)
    T = float(input_dict["T"])
    dt = T / steps
    f = torch.fft.rfft2(fields)
    obs = torch.zeros((2, steps), dtype=torch.float64, device=device)
    for i in range(steps):
        obs[:, i] = compute_observables(f, param_dict)
        f = integrate(f, dt, 1, param_dict, "TDRK4")
    f_lam = torch.fft.rfft2(laminar_flow(param_dict).to(device=device, dtype=torch.float64))
    return obs / compute_observables(f_lam, param_dict).reshape(2, 1)
