"""Matrix-free GMRES (reference: gmres, jax_scripts/lib/linalg.py:12-98).

The Krylov basis Q and Hessenberg H live on the device in FP64; each Arnoldi
step's modified Gram-Schmidt runs as one thread-block-cluster kernel
(ecs_arnoldi_mgs) and the small least-squares problem as one CTA
(ecs_hessenberg_lstsq).  A and the preconditioners are callables on flat
[T, fields, sx] vectors, as in the reference.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib
from .context import stream_ptr


def _lib_call(name, *args):
    lib = _lib.load()
    _lib.check(getattr(lib, name)(*args))


def gmres(A, b, inner, outer=1, preconditioner_list=()):
    """Returns (x, rel_res) with the reference's semantics: left preconditioners
    applied in order, MGS Arnoldi without re-orthogonalisation, no restarts
    (`outer` is accepted and unused, as in linalg.py:12-98)."""
    b = b.to(torch.float64).contiguous()
    n = b.numel()
    dev = b.device

    def precond(v):
        for M in preconditioner_list:
            v = M(v)
        return v

    Q = torch.zeros((inner + 1, n), dtype=torch.float64, device=dev)   # column-major basis, ld = n
    H = torch.zeros((inner, inner + 1), dtype=torch.float64, device=dev)   # column-major (inner+1) x inner
    h0 = torch.zeros(inner + 2, dtype=torch.float64, device=dev)
    b = precond(b).to(torch.float64).contiguous()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    _lib_call("ecs_arnoldi_mgs", vp(Q), n, -1, vp(b), vp(h0), n, stream_ptr())   # Q[:,0] = b/|b|
    for k in range(inner):
        Aq = precond(A(Q[k])).to(torch.float64).contiguous()
        col = torch.zeros(inner + 2, dtype=torch.float64, device=dev)
        _lib_call("ecs_arnoldi_mgs", vp(Q), n, k, vp(Aq), vp(col), n, stream_ptr())
        H[k, : min(k + 2, inner + 1)] = col[: min(k + 2, inner + 1)]
    b2 = torch.mv(Q, b)                        # Q^T b   (linalg.py:92)
    y = torch.empty(inner, dtype=torch.float64, device=dev)
    Hc = H.contiguous()
    _lib_call("ecs_hessenberg_lstsq", vp(Hc), inner + 1, inner, vp(b2), vp(y), stream_ptr())
    x = torch.mv(Q[:inner].t(), y)             # Q[:, :inner] y  (linalg.py:94)
    rel_res = torch.linalg.norm(precond(A(x)) - b) / torch.linalg.norm(b)
    return x, rel_res
