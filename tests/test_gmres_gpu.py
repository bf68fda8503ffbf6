"""Device GMRES (MGS Arnoldi + Hessenberg least squares) against the oracle's
numpy restatement of linalg.gmres (jax_scripts/lib/linalg.py:12-98)."""
import numpy as np
import pytest
import torch

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200.linalg import gmres

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,inner,with_pre", [(500, 16, False), (32770, 24, True), (131074, 8, False)])
def test_gmres_matches_oracle(cuda, n, inner, with_pre):
    rng = np.random.default_rng(n)
    # a matrix-free operator (diagonal + low rank) whose spectrum is spread enough
    # that GMRES does not reach Arnoldi breakdown within `inner` steps
    d = 1.0 + 99.0 * rng.random(n)
    U = rng.standard_normal((n, 3)) / np.sqrt(n)
    V = rng.standard_normal((n, 3))
    b = rng.standard_normal(n)
    A_np = lambda x: d * x + U @ (V.T @ x)
    AT_np = lambda x: d * x + V @ (U.T @ x)
    dt = lambda a: torch.as_tensor(a, device="cuda")
    dd, Ud, Vd = dt(d), dt(U), dt(V)
    A_t = lambda x: dd * x + Ud @ (Vd.T @ x)
    AT_t = lambda x: dd * x + Vd @ (Ud.T @ x)
    pre_np = [AT_np] if with_pre else []
    pre_t = [AT_t] if with_pre else []
    x_ref, r_ref = O.gmres(A_np, b, inner, 1, pre_np)
    x, r = gmres(A_t, dt(b), inner, 1, pre_t)
    assert np.linalg.norm(x.cpu().numpy() - x_ref) / np.linalg.norm(x_ref) < 1e-10
    assert abs(float(r) - r_ref) <= 1e-9 * max(r_ref, 1e-12) + 1e-14


def test_gmres_converges_on_small_system(cuda):
    n = 200
    rng = np.random.default_rng(1)
    M = np.diag(np.linspace(1.0, 4.0, n)) + rng.standard_normal((n, n)) * 0.01
    b = rng.standard_normal(n)
    Md = torch.as_tensor(M, device="cuda")
    x, r = gmres(lambda v: Md @ v, torch.as_tensor(b, device="cuda"), 24)
    x_ref, r_ref = O.gmres(lambda v: M @ v, b, 24)
    assert float(r) < 1e-8 and abs(float(r) - r_ref) <= 1e-6 * r_ref + 1e-15
    assert np.linalg.norm(x.cpu().numpy() - np.linalg.solve(M, b)) / np.linalg.norm(np.linalg.solve(M, b)) < 1e-7
