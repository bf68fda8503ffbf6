"""DNS data generation (reference: jax_scripts/generate_turbulence.py): a
Lawson-RK6 transient from random data, a series of snapshots, and the
recurrence matrix of their spectral magnitudes, saved in the reference's npz
layout (dictionaryIO.save_dicts)."""

from __future__ import annotations

import numpy as np
import torch

from . import context as _ctx
from .dictionaryIO import save_dicts
from .mhd import make_param_dict
from .timestepping import integrate


def recurrence(fs, param_dict):
    """dist[j, i] = || |fs_j| - |fs_i| ||_2 for snapshots fs [S, 2, n, n//2+1]
    (generate_turbulence.py:136-146), on the device (ecs_recurrence)."""
    n = _ctx.check_spectral(fs, "snapshots")
    if fs.dim() != 4:
        raise ValueError(f"snapshots must be [S, 2, n, n//2+1], got {tuple(fs.shape)}")
    S = fs.shape[0]
    if S == 0:
        return torch.empty((0, 0), dtype=torch.float64, device=fs.device)
    rdt = torch.float64 if fs.dtype == torch.complex128 else torch.float32
    ctx = _ctx.get_context(param_dict, n, rdt, 1)
    fs = fs.contiguous()
    dist = torch.empty((S, S), dtype=torch.float64, device=fs.device)
    ctx.call("ecs_recurrence", _ctx.ptr(fs), S, _ctx.ptr(dist), _ctx.stream_ptr())
    return dist


def generate_turbulence(n=128, dt=1 / 256, ministeps=64, steps=256, transient_steps=1024 * 2 * 4, nu=1 / 40,
                        eta=1 / 40, b0=(0.0, 0.3), seed=111111, amp=10.0, data_type=torch.float64, path=None):
    """generate_turbulence.py:21-162.  Random initial fields amp * N(0, 1) [2, n, n]
    (:53-55; numpy PCG64 seeded with `seed` where the reference draws them with
    jax.random), rfft2 and mask (:77-79); `transient_steps` Lawson-RK6 steps of
    dt (:84-94); `steps` snapshots each `ministeps` steps apart (:101-124); the
    recurrence matrix (:136-146).  With `path`, saves {"fs", "dist"} and the
    parameters as the reference does (:161-162, dictionaryIO.save_dicts).  Returns (fs, dist,
    param_dict); fs is [steps, 2, n, n//2+1] complex on the device."""
    pd = make_param_dict(n, nu, eta, b0=b0, forcing="kolmogorov", data_type=data_type)
    pd.update({"dt": dt, "ministeps": ministeps, "steps": steps})
    rng = np.random.default_rng(seed)
    f = amp * rng.standard_normal((2, n, n))
    ctype = torch.complex128 if data_type == torch.float64 else torch.complex64
    f = torch.as_tensor(np.fft.rfft2(f), dtype=ctype, device="cuda") * pd["mask"].to("cuda")
    if transient_steps > 0:
        # one run of transient_steps steps of h = (dt * transient_steps) / transient_steps
        f = integrate(f, dt * transient_steps, transient_steps, pd, "Lawson_RK6")
    fs = torch.empty((steps, 2, n, n // 2 + 1), dtype=ctype, device="cuda")
    for i in range(steps):
        f = integrate(f, dt * ministeps, ministeps, pd, "Lawson_RK6")   # :105 one_step
        fs[i] = f
    dist = recurrence(fs, pd)
    if path is not None:
        save_dicts(path, {"fs": fs.cpu().numpy(), "dist": dist.cpu().numpy()}, pd)
    return fs, dist, pd
