"""Flat-vector helpers and the Newton line search (reference: jax_scripts/lib/utils.py).

Flat vectors follow jax.flatten_util.ravel_pytree of {"T","fields","sx"}
(sorted keys): [T, fields(2 n^2), sx].
"""

from __future__ import annotations

import torch


def flatten(d):
    """ravel_pytree order [T, fields, sx] of an input or output dict."""
    f = d["fields"]
    T = torch.as_tensor(d["T"], dtype=f.dtype, device=f.device).reshape(1)
    sx = torch.as_tensor(d["sx"], dtype=f.dtype, device=f.device).reshape(1)
    return torch.cat([T, f.reshape(-1), sx])


def unflatten(v, n):
    return {"T": v[0], "fields": v[1:-1].reshape(2, n, n), "sx": v[-1]}


def relative_error_RPO(input_dict, f):
    """|f["fields"]| / |input["fields"]| (jax_scripts/newton.py:141-143)."""
    return torch.linalg.norm(f["fields"]) / torch.linalg.norm(input_dict["fields"])


def line_search_unravel(x, step, obj, unravel_fn, f_vec, max_iters=20):
    """Damped step x - damp*step, halving damp until |obj| decreases
    (jax_scripts/lib/utils.py:17-58); returns (x_final, damp)."""
    norm_orig = torch.linalg.norm(f_vec)
    damp, done = 1.0, False
    for _ in range(max_iters):
        if done:
            break
        x_temp = x - damp * step
        norm_temp = torch.linalg.norm(flatten(obj(unravel_fn(x_temp))))
        improved = bool(norm_temp < norm_orig)
        if improved:
            x = x_temp
        else:
            damp = damp / 2.0
        done = improved
    return x, damp
