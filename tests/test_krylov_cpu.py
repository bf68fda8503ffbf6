"""The oracle's restatements of the reference's alternative solvers
(jax_scripts/lib/linalg.py:100-570) and diagonal estimators
(jax_scripts/lib/preconditioners.py:225-360), checked by their algebra on
small dense problems: exact solves when the Krylov space is the whole space,
the trust-region bound when it binds, exact diagonals of diagonal operators."""
import numpy as np

from oracle import krylov as K


def _problem(n=24, seed=0, shift=3.0):
    rng = np.random.default_rng(seed)
    A = shift * np.eye(n) + rng.standard_normal((n, n)) / np.sqrt(n)
    c = rng.standard_normal(n)
    return A, c


def test_hookstep_v2_full_space_is_newton():
    """f(x) = A x - c; with m = n and a loose bound the step is the Newton step."""
    A, c = _problem()
    n = A.shape[0]
    x = np.zeros(n)
    f = lambda v: A @ v - c
    xn, s, rr = K.newton_gmres_hookstep_v2(lambda v: A @ v, f(x), n, 1e3, f, x)
    assert np.linalg.norm(xn - np.linalg.solve(A, c)) < 1e-10 * np.linalg.norm(xn)
    assert rr < 1e-10 and s == 2e3


def test_hookstep_v2_bound_binds():
    """A tight bound: the regularised Krylov coefficients have 2-norm s, the
    step still lowers |f| (a descent direction), and s doubles on acceptance."""
    A, c = _problem(seed=1)
    n = A.shape[0]
    x = np.zeros(n)
    f = lambda v: A @ v - c
    s0 = 0.3
    xn, s, rr = K.newton_gmres_hookstep_v2(lambda v: A @ v, f(x), 8, s0, f, x)
    assert abs(np.linalg.norm(xn - x) - s0) < 1e-9 * s0   # Q has orthonormal columns
    assert np.linalg.norm(f(xn)) < np.linalg.norm(f(x)) and s == 2 * s0


def test_hookstep_v1_normal_equations():
    A, c = _problem(seed=2)
    n = A.shape[0]
    x = np.zeros(n)
    f = lambda v: A @ v - c
    f0 = f(x)
    xn, s, r1, r2 = K.newton_gmres_hookstep(lambda v: A.T @ (A @ v), A.T @ f0, n, 1e3, f, f0,
                                            lambda v: A @ v, -f0, x)
    assert np.linalg.norm(xn - np.linalg.solve(A, c)) < 1e-9 * np.linalg.norm(xn)
    assert r1 < 1e-9


def test_block_gmres_minimises_over_the_block_space():
    """With b a column of the start block, x minimises |A x - b| over
    span{B, AB, ..., A^(m-1) B}; every singular value of H exceeds 1
    (A = 3 I + noise), so none is left uninverted."""
    A, c = _problem(n=40, seed=3)
    B = np.concatenate([c[:, None], np.random.default_rng(4).standard_normal((40, 3))], axis=1)
    m = 4
    x = K.block_gmres(lambda X: A @ X, c, m, B)
    Kr = np.concatenate([np.linalg.matrix_power(A, j) @ B for j in range(m)], axis=1)
    xs = Kr @ np.linalg.lstsq(A @ Kr, c, rcond=None)[0]
    assert np.linalg.norm(x - xs) < 1e-9 * np.linalg.norm(xs)
    assert np.linalg.norm(A @ x - c) < np.linalg.norm(c)


def test_adjoint_gmres_solves_rectangular_least_squares():
    rng = np.random.default_rng(5)
    A = rng.standard_normal((30, 20))
    b = rng.standard_normal(30)
    x, hist = K.adjoint_GMRES(lambda v: A @ v, lambda v: A.T @ v, b, 30, 20, 20,
                              x0_fn=lambda bb, _: A @ (A.T @ bb))
    xs = np.linalg.lstsq(A, b, rcond=None)[0]
    assert np.linalg.norm(x - xs) < 1e-9 * np.linalg.norm(xs)


def test_adjoint_gmres_outer_restarts_with_preconditioner():
    """Two outer iterations with a diagonal left preconditioner: the residual
    of the preconditioned system falls below that of one iteration."""
    A, c = _problem(n=40, seed=6, shift=1.0)
    d = np.linspace(0.5, 2.0, 40)
    M = lambda v, mode: d * v
    x1, h1 = K.adjoint_GMRES(lambda v: A @ v, lambda v: A.T @ v, c, 40, 40, 10, outer=1, precond_left=[M])
    x2, h2 = K.adjoint_GMRES(lambda v: A @ v, lambda v: A.T @ v, c, 40, 40, 10, outer=2, precond_left=[M])
    assert h2[-1] < h1[-1]


def test_spatial_diagonal_of_a_diagonal_operator_is_exact():
    """z * (D z) = D for +-1 probes: Hutchinson is exact for diagonal D."""
    nf = 2 * 8 * 8
    D = np.random.default_rng(7).standard_normal(nf)
    est = K.diagonal_estimate_spatial(lambda zp: zp[:, 1:-1] * D, nf, k=2, batch=3)
    assert np.allclose(est, D, rtol=0, atol=1e-14)


def test_fourier_diagonal_of_a_fourier_multiplier():
    """For J = irfft2(c rfft2(.)) with a real multiplier c on the interior ky
    columns, every probe gives conj(z) c z = c there."""
    n = 8
    rng = np.random.default_rng(8)
    c = rng.standard_normal((2, n, n // 2 + 1))
    c[..., 0] = 0
    c[..., -1] = 0

    def op(zp):
        zf = zp[:, 1:-1].reshape(-1, 2, n, n)
        return np.fft.irfft2(c * np.fft.rfft2(zf), s=(n, n)).reshape(zf.shape[0], -1)

    est = K.diagonal_estimate_fourier(op, (2, n, n), k=3, batch=2)
    assert np.allclose(est, np.fft.irfft2(c, s=(n, n)), atol=1e-12)
