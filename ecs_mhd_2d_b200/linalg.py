"""Matrix-free Krylov solvers (reference: jax_scripts/lib/linalg.py): gmres,
newton_gmres_hookstep, newton_gmres_hookstep_v2, block_gmres, adjoint_GMRES.

The Krylov bases live on the device in FP64, one vector per row (column-major
with leading dimension len for the kernels); each Arnoldi or Golub-Kahan step's
modified Gram-Schmidt, re-orthogonalisation sweeps included, runs as one
thread-block-cluster kernel (ecs_arnoldi_mgs / ecs_arnoldi_mgs_reorth) and the
GMRES least-squares problem as one CTA (ecs_hessenberg_lstsq).  The projected
problems of the trust-region and bidiagonal solvers (SVD / eigendecomposition
of an (m+1) x m matrix, the scalar bisection on the Lagrange multiplier) are
tiny and sequential and run in FP64 LAPACK on the host.  A and the
preconditioners are callables on flat [T, fields, sx] vectors, as in the
reference.
"""

from __future__ import annotations

import ctypes

import numpy as np
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
    if not 1 <= inner <= 128:
        raise ValueError(f"gmres: inner must be in [1, 128] (the projected solve is one CTA), got {inner}")
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
    _lib_call("ecs_arnoldi_mgs", _vp(Q), n, -1, _vp(b, n), _vp(h0), n, stream_ptr())   # Q[:,0] = b/|b|
    for k in range(inner):
        Aq = precond(A(Q[k])).to(torch.float64).contiguous()
        col = torch.zeros(inner + 2, dtype=torch.float64, device=dev)
        _lib_call("ecs_arnoldi_mgs", _vp(Q), n, k, _vp(Aq, n), _vp(col), n, stream_ptr())
        H[k, : min(k + 2, inner + 1)] = col[: min(k + 2, inner + 1)]
    b2 = torch.mv(Q, b)                        # Q^T b   (linalg.py:92)
    y = torch.empty(inner, dtype=torch.float64, device=dev)
    Hc = H.contiguous()
    _lib_call("ecs_hessenberg_lstsq", _vp(Hc), inner + 1, inner, _vp(b2), _vp(y), stream_ptr())
    x = torch.mv(Q[:inner].t(), y)             # Q[:, :inner] y  (linalg.py:94)
    rel_res = torch.linalg.norm(precond(A(x)) - b) / torch.linalg.norm(b)
    return x, rel_res


def _vp(t, numel=None):
    """Device pointer of a contiguous FP64 CUDA tensor; with `numel`, the
    tensor must hold exactly that many values (a Krylov vector of the basis's
    length), since the kernels read as many as the basis is long."""
    if not (t.is_cuda and t.is_contiguous() and t.dtype == torch.float64):
        raise ValueError(f"Krylov vectors must be contiguous FP64 CUDA tensors, got {t.dtype} on {t.device}")
    if numel is not None and t.numel() != numel:
        raise ValueError(f"vector has {t.numel()} values, the Krylov basis has length {numel}")
    return ctypes.c_void_p(t.data_ptr())


def _orth(Q, k, w, hcol, reorth):
    """MGS of w against rows 0..k of Q with `reorth` extra sweeps; row k+1 of Q
    receives w/|w|, hcol[0..k] the first sweep's projections, hcol[k+1] = |w|."""
    n = Q.shape[1]
    w = w.to(torch.float64).contiguous()
    if not (-1 <= k < Q.shape[0] - 1) or hcol.numel() < k + 2:
        raise ValueError(f"_orth: step {k} outside a basis of {Q.shape[0]} vectors (or hcol too short)")
    _lib_call("ecs_arnoldi_mgs_reorth", _vp(Q), n, k, _vp(w, n), _vp(hcol), n, reorth, stream_ptr())


def _bisection(g, lower, upper, maxit):
    """linalg.py:165-177 / :289-301."""
    if g(0) > 0:
        return 0
    t = 0
    for _ in range(maxit):
        t = (lower + upper) / 2
        if g(t) > 0:
            upper = t
        else:
            lower = t
    return t


def _flat_objective(objective, n):
    from .utils import flatten, unflatten
    return lambda x: flatten(objective(unflatten(x, n)))


def newton_gmres_hookstep(AtA, Atb, m, s, f, f0, J, b, input_dict, max_halvings=200):
    """Newton step from the Krylov space of A^T A with a bound s on its 2-norm
    (linalg.py:100-213): Arnoldi with two re-orthogonalisation sweeps,
    eigendecomposition of the (symmetrised, as jnp.linalg.eigh does) m x m H,
    bisection on the Lagrange multiplier, s halved until |f(x - step)| < |f0|
    and then doubled.  f maps input dicts to output dicts.  Returns
    (input_dict, s, rel_res_1, rel_res_2).  Where the reference loops for ever
    when no step decreases |f|, this raises after `max_halvings` halvings."""
    from .utils import flatten, unflatten
    Atb = Atb.to(torch.float64).contiguous()
    nv = Atb.numel()
    Q = torch.zeros((m + 1, nv), dtype=torch.float64, device=Atb.device)
    H = np.zeros((m, m))
    col = torch.zeros(m + 2, dtype=torch.float64, device=Atb.device)
    _orth(Q, -1, Atb, col, 0)                                            # :130
    for k in range(m):                                                   # :138-153
        _orth(Q, k, AtA(Q[k]), col, 2)
        c = col.cpu().numpy()
        H[: k + 1, k] = c[: k + 1]
        if k != m - 1:
            H[k + 1, k] = c[k + 1]
    b2 = torch.mv(Q[:m], Atb).cpu().numpy()                              # :156
    D, V = np.linalg.eigh((H + H.T) / 2)                                 # :159
    b2 = V.T @ b2                                                        # :162
    x0 = flatten(input_dict).to(torch.float64)
    n = input_dict["fields"].shape[-1]
    f_vector = _flat_objective(f, n)
    nb, nf0 = float(torch.linalg.norm(b)), float(torch.linalg.norm(f0))
    for _ in range(max_halvings):                                        # :185-203
        g = lambda t: s - np.linalg.norm(b2 / (D + t))
        t = 0 if g(0) > 0 else _bisection(g, 0, nb / s, 128)
        coef = torch.as_tensor(V @ (b2 / (D + t)), device=Q.device)
        step = torch.mv(Q[:m].t(), coef)
        if float(torch.linalg.norm(f_vector(x0 - step))) < nf0:
            s = s * 2
            break
        s = s / 2
    else:
        raise RuntimeError("newton_gmres_hookstep: no step decreased |f|")
    rel_res_1 = torch.linalg.norm(AtA(step) - Atb) / torch.linalg.norm(Atb)   # :206
    rel_res_2 = torch.linalg.norm(J(step) + b) / torch.linalg.norm(b)         # :207-208
    return unflatten(x0 - step, n), s, rel_res_1, rel_res_2


def newton_gmres_hookstep_v2(A, b, m, s, objective, input_dict, max_halvings=200):
    """Newton-GMRES step with a bound s on its 2-norm (linalg.py:217-337):
    Arnoldi with two re-orthogonalisation sweeps (one cluster kernel per
    step), SVD of the (m+1) x m H, the regularised solution when |y| > s*s
    (the reference's test), s halved until |objective(x - dx)| < |b| and then
    doubled.  Returns (input_dict, s, rel_res).  Where the reference loops for
    ever when no step decreases the objective, this raises after
    `max_halvings` halvings."""
    from .utils import flatten, unflatten
    b = b.to(torch.float64).contiguous()
    nv = b.numel()
    Q = torch.zeros((m + 1, nv), dtype=torch.float64, device=b.device)
    H = np.zeros((m + 1, m))
    col = torch.zeros(m + 2, dtype=torch.float64, device=b.device)
    _orth(Q, -1, b, col, 0)                                              # :247
    for k in range(m):                                                   # :254-266
        _orth(Q, k, A(Q[k]), col, 2)
        H[: k + 2, k] = col[: k + 2].cpu().numpy()
    b2 = torch.mv(Q, b).cpu().numpy()                                    # :269
    U, S, Vh = np.linalg.svd(H, full_matrices=False)                     # :272
    y = Vh.T @ ((U.T @ b2) / S)                                          # :275-277
    x = flatten(input_dict).to(torch.float64)
    n = input_dict["fields"].shape[-1]
    f = _flat_objective(objective, n)
    nb = float(torch.linalg.norm(b))
    for _ in range(max_halvings):                                        # :281-329
        if np.linalg.norm(y) > s * s:
            b4 = Vh @ (H.T @ b2)
            g = lambda t: s - np.linalg.norm(b4 / (S * S + t))
            t = _bisection(g, 0, np.sqrt(m) * np.linalg.norm(b4) / s, 128)
            y = Vh.T @ (b4 / (S * S + t))
        dx = torch.mv(Q[:-1].t(), torch.as_tensor(y, device=Q.device))  # :312
        if float(torch.linalg.norm(f(x - dx))) < nb:
            s = s * 2
            break
        s = s / 2
    else:
        raise RuntimeError("newton_gmres_hookstep_v2: no step decreased the objective")
    rel_res = torch.linalg.norm(A(dx) - b) / torch.linalg.norm(b)       # :332
    return unflatten(x - dx, n), s, rel_res


def block_gmres(A, b, m, B, tol=1e-8, iteration=0):
    """Block Krylov solve of A x = b (linalg.py:340-427) over the space
    {B, AB, ..., A^m B}: A maps an [n, s] block to [n, s], e.g. one batched
    JVP of s tangents.  Each new column is orthogonalised against all previous
    basis vectors by the cluster kernel, its normalised copy is the next
    block's column, and the basis vector itself gets one more sweep (not
    renormalised); singular values of H below 1 are not inverted."""
    b = b.to(torch.float64)
    nv, sb = B.shape
    dev = B.device
    Q = torch.zeros((sb * (m + 1), nv), dtype=torch.float64, device=dev)
    H = np.zeros((sb * (m + 1), sb * m))
    Bq = torch.linalg.qr(B.to(torch.float64), mode="reduced")[0]         # :369
    Q[:sb] = Bq.t()                                                      # :372
    Bk = Bq
    col = torch.zeros(sb * (m + 1) + 1, dtype=torch.float64, device=dev)
    tmp = torch.empty(nv, dtype=torch.float64, device=dev)
    for k in range(m):                                                   # :375
        C = A(Bk).to(torch.float64).clone()                              # :377
        for i in range(sb):                                              # :380
            a = k * sb + i
            w = C[:, i].contiguous()
            _orth(Q, a + sb - 1, w, col, 0)                              # :384-390, row a+sb = w/|w|
            c = col[: a + sb + 1].cpu().numpy()
            H[: a + sb, a] = c[: a + sb]
            if c[a + sb] < tol:                                          # :393-396
                Q[a + sb].zero_()
                for j in range(a + sb):                                  # the unnormalised residual
                    w = w - torch.dot(Q[j], w) * Q[j]
                C[:, i] = w
                break
            H[a + sb, a] = c[a + sb]                                     # :398
            C[:, i] = Q[a + sb]                                          # :400
            tmp.copy_(Q[a + sb])
            _orth(Q, a + sb - 1, tmp, col, 0)                            # :404-406 (one more sweep)
            Q[a + sb] *= col[a + sb]                                     # ... not renormalised
        Bk = C                                                           # :407
    b2 = torch.mv(Q, b).cpu().numpy()                                    # :412
    U, sv, Vh = np.linalg.svd(H, full_matrices=False)                    # :414
    inv_s = 1 / sv
    inv_s[sv < 1.0] = 1                                                  # :417-421
    y = Vh.T @ ((U.T @ b2) * inv_s)                                      # :416-424
    return torch.mv(Q[: y.shape[0]].t(), torch.as_tensor(y, device=dev))   # :426


def adjoint_GMRES(A, A_t, b, m, n, inner, outer=1, precond_left=(), x0_fn=lambda x, _: x, seed=0, verbose=False):
    """Least-squares solve of A x = b by Golub-Kahan bidiagonalisation
    (linalg.py:431-570): A maps length-n vectors to length-m, A_t the reverse
    (e.g. the VJP); left preconditioners M(x, "no_trans" | "trans").  Both
    orthogonalisations (with two re-orthogonalisation sweeps) are one cluster
    kernel each; B is filled in the reference's assignment order and solved by
    SVD least squares (lstsq, rcond=None) on the host.  x0_fn(b, rng) gets
    numpy.random.default_rng([seed, outer_iteration]) where the reference
    passes a jax.random key.  Returns x."""
    b = b.to(torch.float64).contiguous()
    dev = b.device
    Bm = np.zeros((inner + 1, inner))
    U = torch.zeros((inner + 1, m), dtype=torch.float64, device=dev)
    V = torch.zeros((inner + 1, n), dtype=torch.float64, device=dev)   # one spare row for the kernel
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    b0 = b.clone()                                                       # :479
    for M in precond_left:                                               # :482-483
        b = M(b, "no_trans")
    col = torch.zeros(inner + 2, dtype=torch.float64, device=dev)
    for it in range(outer):                                              # :488
        x0 = x0_fn(b, np.random.default_rng([seed, it]))                 # :490-493
        _orth(U, -1, x0, col, 0)                                         # :496
        for i in range(inner):                                           # :499
            Au = U[i]
            for M in reversed(precond_left):                             # :502-505
                Au = M(Au, "trans")
            Au = A_t(Au)
            _orth(V, i - 1, Au, col, 2)                                  # :508-521
            c = col[: i + 1].cpu().numpy()
            Bm[i, :i] = c[:i]
            Bm[i, i] = c[i]
            Av = A(V[i])                                                 # :524-526
            for M in precond_left:
                Av = M(Av, "no_trans")
            _orth(U, i, Av, col, 2)                                      # :529-540
            c = col[: i + 2].cpu().numpy()
            Bm[: i + 1, i] = c[: i + 1]
            Bm[i + 1, i] = c[i + 1]
        b2 = torch.mv(U, b).cpu().numpy()                                # :544
        projection_b = np.linalg.norm(b2) / float(torch.linalg.norm(b))  # :547
        y = np.linalg.lstsq(Bm, b2, rcond=None)[0]                       # :551
        x = x + torch.mv(V[:inner].t(), torch.as_tensor(y, device=dev))  # :554-557
        Ax = A(x)                                                        # :560-562
        for M in precond_left:
            Ax = M(Ax, "no_trans")
        b = b0 - Ax                                                      # :563
        rel_res = float(torch.linalg.norm(b) / torch.linalg.norm(b0))    # :565
        if verbose:
            print(f"outer iter {it:03d}: relative residual = {rel_res:.6e}, |b2|/|b|={projection_b:.6e}")
    return x
