"""Grid tables and the MHD right-hand side (reference: jax_scripts/lib/mhd_jax.py).

``construct_domain`` and ``dissipation`` build small host-side tables exactly as
the reference does; ``state_vel`` runs the fused sm_100a kernels through the C-ABI.
"""

from __future__ import annotations

import numpy as np
import torch

from . import context as _ctx

PI_LITERAL = 3.14159265358979323846  # mhd_jax.py:47


def _device():
    return torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")


def construct_domain(n: int, data_type=torch.float64):
    """Grid dictionary of mhd_jax.construct_domain (mhd_jax.py:20-94).

    Returns torch tensors: x, y [n,n]; kx, ky, mask, to_u, to_v, inv_lap
    [n, n//2+1] with kx, ky, to_u, to_v pre-masked (mhd_jax.py:87-90)."""
    assert data_type in (torch.float32, torch.float64)
    npdt = np.float64 if data_type == torch.float64 else np.float32
    grid = np.arange(n, dtype=npdt) / n * 2 * PI_LITERAL
    x, y = np.meshgrid(grid, grid, indexing="ij")
    k = np.fft.fftfreq(n, d=1 / n).astype(npdt)
    kx = k.reshape(-1, 1)
    ky = k[: n // 2 + 1].reshape(1, -1)
    mask = (np.abs(kx) < n / 3) & (np.abs(ky) < n / 3)
    mask[0, 0] = False
    k_sq = kx * kx + ky * ky
    k_sq[0, 0] = 1
    inv_lap = -1 / k_sq
    inv_lap[0, 0] = 0
    inv_lap = inv_lap * mask
    to_u = ky / k_sq
    to_v = -kx / k_sq
    kx, ky, to_u, to_v = kx * mask, ky * mask, to_u * mask, to_v * mask
    dev = _device()
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    return {"x": t(x), "y": t(y), "kx": t(kx), "ky": t(ky), "mask": t(mask), "to_u": t(to_u),
            "to_v": t(to_v), "inv_lap": t(inv_lap)}


def make_param_dict(n, nu, eta, b0=(0.0, 0.1), forcing="kolmogorov", data_type=torch.float64, **extra):
    """construct_domain + physics, as dictionaryIO.recompute_grid_information does
    (jax_scripts/lib/dictionaryIO.py:64-78).  ``forcing`` is "kolmogorov"
    (-4cos(4y), the reference solutions' forcing_str), "kolmogorov+" (+4cos(4y)),
    a callable f(x, y) on numpy grids, or an [n, n] array."""
    pd = construct_domain(n, data_type)
    grid = np.arange(n, dtype=np.float64) / n * 2 * PI_LITERAL
    xg, yg = np.meshgrid(grid, grid, indexing="ij")
    if isinstance(forcing, str):
        amp = {"kolmogorov": -4.0, "kolmogorov+": 4.0}[forcing]
        fr = amp * np.cos(4 * yg)
    elif callable(forcing):
        fr = np.asarray(forcing(xg, yg), dtype=np.float64)
    else:
        fr = np.asarray(forcing.detach().cpu() if isinstance(forcing, torch.Tensor) else forcing, np.float64)
    pd.update({"nu": float(nu), "eta": float(eta), "b0": [float(b0[0]), float(b0[1])],
               "forcing": torch.as_tensor(fr.astype(np.float64 if data_type == torch.float64 else np.float32),
                                          device=pd["x"].device)})
    pd.update(extra)
    return pd


def dissipation(param_dict):
    """L = -(kx^2+ky^2)[nu, eta] of shape [2, n, n//2+1] (mhd_jax.py:97-102)."""
    k_sq = param_dict["kx"] ** 2 + param_dict["ky"] ** 2
    coeffs = torch.tensor([param_dict["nu"], param_dict["eta"]], dtype=k_sq.dtype, device=k_sq.device)
    return -k_sq * coeffs.reshape(2, 1, 1)


def state_vel(fields, param_dict, include_dissipation):
    """Time derivative of the rfft2 state [..., 2, n, n//2+1] (mhd_jax.py:105-175),
    computed by the fused column/row kernels (ecs_state_vel)."""
    n = _ctx.check_spectral(fields, "state_vel input")
    rdt = torch.float64 if fields.dtype == torch.complex128 else torch.float32
    lead = fields.shape[:-3]
    f = fields.reshape(-1, 2, n, n // 2 + 1).contiguous()
    B = f.shape[0]
    if B == 0:
        return torch.empty_like(fields)
    ctx = _ctx.get_context(param_dict, n, rdt, B)
    out = torch.empty_like(f)
    ctx.call("ecs_state_vel", _ctx.ptr(f), _ctx.ptr(out), B, int(bool(include_dissipation)), _ctx.stream_ptr())
    return out.reshape(*lead, 2, n, n // 2 + 1)
