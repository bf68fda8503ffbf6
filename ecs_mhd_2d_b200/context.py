"""Device contexts (grid tables + workspace) keyed by the static physics parameters.

A context is the C-ABI ``ecs_ctx``; it replaces the grid arrays that the
reference keeps in ``param_dict`` (jax_scripts/lib/mhd_jax.py:20-94) with device
tables and preallocated workspace for a maximum batch.
"""

from __future__ import annotations

import ctypes
import hashlib
import itertools

import numpy as np
import torch

from . import _lib

_CACHE = {}


def torch_dtype_code(dt):
    if dt == torch.float64:
        return _lib.ECS_F64
    if dt == torch.float32:
        return _lib.ECS_F32
    raise TypeError(f"fields must be float64 or float32, got {dt}")


def complex_of(dt):
    return torch.complex128 if dt == torch.float64 else torch.complex64


def stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t: torch.Tensor):
    if not t.is_cuda:
        raise ValueError("tensor must live on the GPU")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return ctypes.c_void_p(t.data_ptr())


# Shape checks run on the host before any pointer reaches a kernel: the
# kernels take sizes from the context (n) and the call (batch), so a tensor
# of another shape would be read or written past its end.

def check_fields(f, what="fields", n=None):
    """A real state [2, n, n] or a batch [B, 2, n, n]; with `n`, of that side."""
    if f.dim() not in (3, 4) or f.shape[-3] != 2 or f.shape[-1] != f.shape[-2]:
        raise ValueError(f"{what} must be [2, n, n] or [B, 2, n, n], got {tuple(f.shape)}")
    if n is not None and f.shape[-1] != n:
        raise ValueError(f"{what} has grid side {f.shape[-1]}, the primal has {n}")


def check_spectral(f, what="state"):
    """rfft2 coefficients [..., 2, n, n//2+1] (complex); returns n."""
    if not torch.is_complex(f):
        raise TypeError(f"{what} must be the rfft2 coefficients (complex), got {f.dtype}")
    if f.dim() < 3 or f.shape[-3] != 2 or f.shape[-1] != f.shape[-2] // 2 + 1:
        raise ValueError(f"{what} must be [..., 2, n, n//2+1], got {tuple(f.shape)}")
    return f.shape[-2]


_GENERATION = itertools.count(1)


class Context:
    """Owns one ``ecs_ctx`` for (device, n, dtype, nu, eta, b0, forcing).

    ``generation`` is unique to each native context this process creates
    (growing the batch re-creates it, dropping any linearisation it held;
    the freed handle's address may come back for the new one)."""

    def __init__(self, n, dtype, nu, eta, b0, forcing=None, max_batch=1):
        if not torch.cuda.is_available():
            raise _lib.EcsError(2, "CUDA device required (no CPU fallback)")
        self.lib = _lib.load()
        self.n, self.dtype = int(n), dtype
        self.code = torch_dtype_code(dtype)
        self.nu, self.eta, self.b0 = float(nu), float(eta), (float(b0[0]), float(b0[1]))
        self.device = torch.cuda.current_device()
        self._forcing = None if forcing is None else np.ascontiguousarray(forcing, dtype=np.float64)
        self.handle = None
        self.max_batch = 0
        self._create(max(1, int(max_batch)))

    def _create(self, max_batch):
        self.close()
        prm = _lib.EcsParams()
        prm.nu, prm.eta = self.nu, self.eta
        prm.b0x, prm.b0y = self.b0
        if self._forcing is not None:
            prm.forcing = self._forcing.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        else:
            prm.forcing = None
            prm.kolmogorov_amp, prm.kolmogorov_k = -4.0, 4
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.ecs_ctx_create(self.n, self.code, ctypes.byref(prm), max_batch, ctypes.byref(h)))
        self.handle = h
        self.generation = next(_GENERATION)
        # the native context holds one linearisation (trajectory record); this
        # token names the Objective call that made the current one
        self.lin_token = None
        self.max_batch = max_batch
        K, M = ctypes.c_int(), ctypes.c_int()
        _lib.check(self.lib.ecs_box_dims(self.handle, ctypes.byref(K), ctypes.byref(M)), self.handle)
        self.K, self.M = K.value, M.value

    def ensure_batch(self, batch):
        if batch > self.max_batch:
            torch.cuda.synchronize()
            self._create(max(batch, 2 * self.max_batch))

    def close(self):
        if getattr(self, "handle", None):
            torch.cuda.synchronize()
            self.lib.ecs_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def call(self, name, *args):
        fn = getattr(self.lib, name)
        _lib.check(fn(self.handle, *args), self.handle)


def _forcing_key(forcing):
    if forcing is None:
        return None
    a = np.ascontiguousarray(forcing.detach().cpu().numpy() if isinstance(forcing, torch.Tensor) else forcing,
                             dtype=np.float64)
    return hashlib.sha1(a.tobytes()).hexdigest(), a


def physics_key(param_dict):
    """(nu, eta, b0, forcing digest): what a context fixes besides grid and dtype."""
    fk = _forcing_key(param_dict.get("forcing"))
    return (float(param_dict["nu"]), float(param_dict["eta"]), float(param_dict["b0"][0]),
            float(param_dict["b0"][1]), None if fk is None else fk[0])


def get_context(param_dict, n, dtype, batch=1):
    """Context for the physics in ``param_dict`` (nu, eta, b0, forcing)."""
    fk = _forcing_key(param_dict.get("forcing"))
    if fk is not None and fk[1].size != int(n) * int(n):
        raise ValueError(f"param_dict['forcing'] has shape {fk[1].shape}, the fields are {n}x{n}")
    key = (torch.cuda.current_device(), int(n), dtype, float(param_dict["nu"]), float(param_dict["eta"]),
           float(param_dict["b0"][0]), float(param_dict["b0"][1]), None if fk is None else fk[0])
    ctx = _CACHE.get(key)
    if ctx is None:
        ctx = Context(n, dtype, param_dict["nu"], param_dict["eta"], param_dict["b0"],
                      None if fk is None else fk[1], max_batch=batch)
        _CACHE[key] = ctx
    ctx.ensure_batch(batch)
    return ctx


def clear_cache():
    for c in list(_CACHE.values()):
        c.close()
    _CACHE.clear()
