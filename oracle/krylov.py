"""CPU restatement of the reference's alternative Krylov / Newton solvers and
diagonal estimators -- TEST INFRASTRUCTURE ONLY (the checker for
``ecs_mhd_2d_b200.linalg`` and ``ecs_mhd_2d_b200.preconditioners``).

Everything acts on flat FP64 numpy vectors and callables, in the order of the
reference's statements (jax_scripts/lib/linalg.py, jax_scripts/lib/
preconditioners.py).  Where the reference draws random numbers with
jax.random, these functions take the numpy generator the device version uses,
so both sides see the same vectors.  Parity unpinned at the value level: the
reference's tests hold no solver outputs, so these are checked by their
algebraic properties (tests/test_oracle_cpu.py).
"""

from __future__ import annotations

import numpy as np


def _bisection(g, lower, upper, maxit):
    """linalg.py:165-177 / :289-301: t = 0 when g(0) > 0, else maxit halvings."""
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


def _mgs(Q, cols, w, reorth):
    """h_j = <w, Q[:,j]>, w -= h_j Q[:,j] for j in cols, then `reorth` more sweeps."""
    h = np.zeros(len(cols))
    for a, j in enumerate(cols):
        h[a] = np.dot(w, Q[:, j])
        w = w - h[a] * Q[:, j]
    for _ in range(reorth):
        for j in cols:
            w = w - np.dot(w, Q[:, j]) * Q[:, j]
    return h, w


def newton_gmres_hookstep(AtA, Atb, m, s, f_vector, f0, J, b, x0, max_halvings=None):
    """linalg.py:100-214 on flat vectors: Arnoldi on A^T A with two
    re-orthogonalisation sweeps, eigendecomposition of the symmetrised m x m H
    (jnp.linalg.eigh symmetrises its input), bisection on the Lagrange
    multiplier, halve/double s.  Returns (x_new, s, rel_res_1, rel_res_2)."""
    n = Atb.size
    Q = np.zeros((n, m))
    H = np.zeros((m, m))
    Q[:, 0] = Atb / np.linalg.norm(Atb)                               # :130
    for k in range(m):                                                # :138
        Aq = AtA(Q[:, k])
        h, Aq = _mgs(Q, range(k + 1), Aq, 2)                          # :141-148
        H[: k + 1, k] = h
        if k != m - 1:                                                # :150-153
            hk1 = np.linalg.norm(Aq)
            H[k + 1, k] = hk1
            Q[:, k + 1] = Aq / hk1
    b2 = Q.T @ Atb                                                    # :156
    D, V = np.linalg.eigh((H + H.T) / 2)                              # :159 (eigh symmetrises)
    b2 = V.T @ b2                                                     # :162
    it = 0
    while True:                                                       # :185
        g = lambda t: s - np.linalg.norm(b2 / (D + t))                # :187
        t = 0 if g(0) > 0 else _bisection(g, 0, np.linalg.norm(b) / s, 128)   # :190
        step = Q @ (V @ (b2 / (D + t)))                               # :193
        f2 = f_vector(x0 - step)                                      # :196
        if np.linalg.norm(f2) < np.linalg.norm(f0):                   # :198
            s = s * 2
            break
        s = s / 2                                                     # :203
        it += 1
        if max_halvings is not None and it >= max_halvings:
            raise RuntimeError("hookstep: no decrease")
    rel_res_1 = np.linalg.norm(AtA(step) - Atb) / np.linalg.norm(Atb)   # :206
    rel_res_2 = np.linalg.norm(J(step) + b) / np.linalg.norm(b)         # :207-208
    return x0 - step, s, rel_res_1, rel_res_2


def newton_gmres_hookstep_v2(A, b, m, s, f_vector, x, max_halvings=None):
    """linalg.py:217-337 on flat vectors: GMRES Arnoldi with two
    re-orthogonalisation sweeps, SVD of the (m+1) x m H, and a 2-norm bound on
    the step found by bisection when |y| > s*s (the reference's test); halve s
    until |f(x - dx)| < |b|, then double it.  Returns (x_new, s, rel_res)."""
    n = b.size
    Q = np.zeros((n, m + 1))
    H = np.zeros((m + 1, m))
    Q[:, 0] = b / np.linalg.norm(b)                                   # :247
    for k in range(m):                                                # :255
        Aq = A(Q[:, k])
        h, Aq = _mgs(Q, range(k + 1), Aq, 2)                          # :256-262
        H[: k + 1, k] = h
        hk1 = np.linalg.norm(Aq)                                      # :264-266
        H[k + 1, k] = hk1
        Q[:, k + 1] = Aq / hk1
    b2 = Q.T @ b                                                      # :269
    U, S, Vh = np.linalg.svd(H, full_matrices=False)                  # :272
    y = Vh.T @ ((U.T @ b2) / S)                                       # :275-277
    it = 0
    while True:                                                       # :281
        if np.linalg.norm(y) > s * s:                                 # :282
            b3 = H.T @ b2                                             # :284
            b4 = Vh @ b3
            g = lambda t: s - np.linalg.norm(b4 / (S * S + t))        # :287
            t = _bisection(g, 0, np.sqrt(m) * np.linalg.norm(b4) / s, 128)   # :303-305
            z = b4 / (S * S + t)                                      # :307
            y = Vh.T @ z                                              # :309
        dx = Q[:, :-1] @ y                                            # :312
        f_new = f_vector(x - dx)                                      # :320
        if np.linalg.norm(f_new) < np.linalg.norm(b):                 # :322
            s = s * 2
            break
        s = s / 2                                                     # :329
        it += 1
        if max_halvings is not None and it >= max_halvings:
            raise RuntimeError("hookstep: no decrease")
    rel_res = np.linalg.norm(A(dx) - b) / np.linalg.norm(b)           # :332
    return x - dx, s, rel_res


def block_gmres(A, b, m, B, tol=1e-8, Bq=None):
    """linalg.py:340-427: block Krylov space {B, AB, ..., A^m B}; A maps an
    [n, s] block to [n, s].  MGS per column against all previous basis vectors,
    one re-orthogonalisation of the new vector (not renormalised), SVD of H
    with singular values below 1 left uninverted.  `Bq` replaces the reduced
    QR of B (so that both sides start from the same orthonormal block)."""
    n, s = B.shape
    Q = np.zeros((n, s * (m + 1)))
    H = np.zeros((s * (m + 1), s * m))
    B = np.linalg.qr(B, mode="reduced")[0] if Bq is None else Bq      # :369
    Q[:, 0:s] = B                                                     # :372
    for k in range(m):                                                # :375
        C = A(B).copy()                                               # :377
        for i in range(s):                                            # :380
            a = k * s + i
            for j in range(a + s):                                    # :384-390
                h = np.dot(Q[:, j], C[:, i])
                H[j, a] = h
                C[:, i] = C[:, i] - h * Q[:, j]
            h = np.linalg.norm(C[:, i])                               # :393
            if h < tol:
                break
            H[a + s, a] = h                                           # :398
            Q[:, a + s] = C[:, i] / h
            C[:, i] = C[:, i] / h
            for j in range(a + s):                                    # :404-406
                h = np.dot(Q[:, j], Q[:, a + s])
                Q[:, a + s] = Q[:, a + s] - h * Q[:, j]
        B = C                                                         # :407
    b2 = Q.T @ b                                                      # :412
    U, sv, Vh = np.linalg.svd(H, full_matrices=False)                 # :414
    b2 = U.T @ b2
    inv_s = 1 / sv
    inv_s[sv < 1.0] = 1                                               # :420-421
    y = Vh.T @ (b2 * inv_s)                                           # :423-424
    return Q[:, : y.shape[0]] @ y                                     # :426


def adjoint_GMRES(A, A_t, b, m, n, inner, outer=1, precond_left=(), x0_fn=lambda x, _: x, seed=0):
    """linalg.py:431-570: Golub-Kahan bidiagonalisation with two
    re-orthogonalisation sweeps on each side, B filled in the reference's
    assignment order, least squares by SVD (lstsq, rcond=None); the residual
    restarts from b0 - M A x.  x0_fn(b, rng) with rng =
    numpy.random.default_rng([seed, outer_iteration])."""
    B = np.zeros((inner + 1, inner))
    U = np.zeros((m, inner + 1))
    V = np.zeros((n, inner))
    x = np.zeros(n)
    b0 = b.copy()                                                     # :479
    for M in precond_left:                                            # :482
        b = M(b, "no_trans")
    history = []
    for it in range(outer):                                           # :488
        x0 = x0_fn(b, np.random.default_rng([seed, it]))              # :490-493
        U[:, 0] = x0 / np.linalg.norm(x0)                             # :496
        for i in range(inner):                                        # :499
            Au = U[:, i]
            for M in reversed(precond_left):
                Au = M(Au, "trans")
            Au = A_t(Au)                                              # :502-505
            h, Au = _mgs(V, range(i), Au, 2)                          # :508-517
            B[i, :i] = h
            B[i, i] = np.linalg.norm(Au)                              # :520
            V[:, i] = Au / B[i, i]
            Av = A(V[:, i])                                           # :524
            for M in precond_left:
                Av = M(Av, "no_trans")
            h, Av = _mgs(U, range(i + 1), Av, 2)                      # :529-537
            B[: i + 1, i] = h
            B[i + 1, i] = np.linalg.norm(Av)                          # :539
            U[:, i + 1] = Av / B[i + 1, i]
        b2 = U.T @ b                                                  # :544
        y = np.linalg.lstsq(B, b2, rcond=None)[0]                     # :551
        x = x + V @ y                                                 # :554-557
        Ax = A(x)                                                     # :560-562
        for M in precond_left:
            Ax = M(Ax, "no_trans")
        b = b0 - Ax                                                   # :563
        history.append(np.linalg.norm(b) / np.linalg.norm(b0))        # :565
    return x, history


def rademacher(rng, shape):
    """+-1 with probability 1/2 (preconditioners.py:232-234)."""
    return 2.0 * (rng.random(shape) < 0.5).astype(np.float64) - 1.0


def diagonal_estimate_spatial(lin_op_fields, nf, k=8, batch=4, seed=0):
    """preconditioners.py:225-263: Hutchinson estimate of the diagonal of the
    fields block of J; lin_op_fields maps a [batch, 2+nf] block of padded
    vectors [0, z, 0] to the [batch, nf] fields block of J z."""
    rng = np.random.default_rng(seed)
    diag = np.zeros(nf)
    for _ in range(k):                                                # :243
        z = rademacher(rng, (batch, nf))                              # :249
        z_pad = np.pad(z, ((0, 0), (1, 1)))                           # :252
        diag += np.sum(z * lin_op_fields(z_pad), axis=0)              # :258
    return diag / k / batch                                           # :263


def diagonal_estimate_fourier(lin_op_fields, shape, k=8, batch=4, seed=0):
    """preconditioners.py:291-348: the same estimate in the rfft2 basis with
    unit-modulus random phases (of the rfft2 of Gaussian fields); returns the
    real-space diagonal irfft2(mean(conj(z) rfft2(J irfft2(z))))."""
    rng = np.random.default_rng(seed)
    nf = int(np.prod(shape))
    diag = 0
    for _ in range(k):                                                # :323
        z = np.fft.rfft2(rng.standard_normal((batch,) + tuple(shape)))   # :306-311
        z = z / np.abs(z)
        z_real = np.fft.irfft2(z, s=shape[-2:]).reshape(batch, nf)    # :328-329
        z_pad = np.pad(z_real, ((0, 0), (1, 1)))                      # :332
        Jz = lin_op_fields(z_pad).reshape((batch,) + tuple(shape))    # :336-338
        Jz = np.fft.rfft2(Jz)
        diag = diag + np.sum(np.conj(z) * Jz, axis=0)                 # :339
    diag = diag / k / batch                                           # :345
    return np.fft.irfft2(diag, s=shape[-2:])                          # :348
