"""The reference's alternative solvers (jax_scripts/lib/linalg.py:100-570) and
diagonal estimators (jax_scripts/lib/preconditioners.py:225-360) on the device
against the oracle's restatements: dense test operators (same matrices on both
sides) and the MHD objective's JVP against torch.func.jvp of the oracle.

Tolerances: 1e-10 relative for dense operators (the cluster kernel's
reductions differ from numpy's in rounding only); 1e-8 for the MHD Newton
steps (JVPs agree to 1e-12, amplified by the Krylov projection)."""
import numpy as np
import pytest
import torch
from torch.func import jvp as tjvp

import oracle as O
from oracle import krylov as K
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import drivers, linalg, preconditioners
from ecs_mhd_2d_b200.synthetic import initial_condition
from ecs_mhd_2d_b200.utils import flatten, unflatten

pytestmark = pytest.mark.gpu
N8 = 8                      # flat length 2 * 8 * 8 + 2 = 130


def _dense(nv, seed, shift=3.0, cols=None):
    rng = np.random.default_rng(seed)
    A = shift * np.eye(nv, cols or nv) + rng.standard_normal((nv, cols or nv)) / np.sqrt(nv)
    return A, rng.standard_normal(nv)


def _rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("s0", [1e3, 0.4])
def test_hookstep_v2_dense_matches_oracle(cuda, s0):
    nv = 2 * N8 * N8 + 2
    A, c = _dense(nv, 1)
    Ad, cd = torch.as_tensor(A, device="cuda"), torch.as_tensor(c, device="cuda")
    objective = lambda d: unflatten(Ad @ flatten(d) - cd, N8)
    x0 = {"fields": torch.zeros(2, N8, N8, dtype=torch.float64, device="cuda"), "T": 0.0, "sx": 0.0}
    b = flatten(objective(x0))
    new, s, rr = linalg.newton_gmres_hookstep_v2(lambda v: Ad @ v, b, 12, s0, objective, x0)
    xo, so, rro = K.newton_gmres_hookstep_v2(lambda v: A @ v, -c, 12, s0, lambda v: A @ v - c, np.zeros(nv))
    assert _rel(flatten(new), xo) < 1e-10 and s == so
    assert abs(float(rr) - rro) <= 1e-10 * rro


def test_hookstep_v1_dense_matches_oracle(cuda):
    nv = 2 * N8 * N8 + 2
    A, c = _dense(nv, 2)
    Ad, cd = torch.as_tensor(A, device="cuda"), torch.as_tensor(c, device="cuda")
    objective = lambda d: unflatten(Ad @ flatten(d) - cd, N8)
    x0 = {"fields": torch.zeros(2, N8, N8, dtype=torch.float64, device="cuda"), "T": 0.0, "sx": 0.0}
    f0 = flatten(objective(x0))
    new, s, r1, r2 = linalg.newton_gmres_hookstep(lambda v: Ad.T @ (Ad @ v), Ad.T @ f0, 10, 0.5, objective, f0,
                                                  lambda v: Ad @ v, -f0, x0)
    xo, so, r1o, r2o = K.newton_gmres_hookstep(lambda v: A.T @ (A @ v), A.T @ -c, 10, 0.5, lambda v: A @ v - c,
                                               -c, lambda v: A @ v, c, np.zeros(nv))
    assert _rel(flatten(new), xo) < 1e-10 and s == so
    assert abs(float(r1) - r1o) <= 1e-9 * r1o and abs(float(r2) - r2o) <= 1e-9 * r2o


def test_block_gmres_dense_matches_oracle(cuda):
    nv = 130
    A, c = _dense(nv, 3)
    B = np.concatenate([c[:, None], np.random.default_rng(4).standard_normal((nv, 5))], axis=1)
    Ad = torch.as_tensor(A, device="cuda")
    x = linalg.block_gmres(lambda X: Ad @ X, torch.as_tensor(c, device="cuda"), 4, torch.as_tensor(B, device="cuda"))
    xo = K.block_gmres(lambda X: A @ X, c, 4, B)
    assert _rel(x, xo) < 1e-10


def test_adjoint_gmres_dense_matches_oracle(cuda):
    """Rectangular 140 x 130 operator, a diagonal left preconditioner, two outer iterations."""
    A, _ = _dense(140, 5, shift=1.0, cols=130)
    b = np.random.default_rng(6).standard_normal(140)
    d = np.linspace(0.5, 2.0, 140)
    Ad, dd = torch.as_tensor(A, device="cuda"), torch.as_tensor(d, device="cuda")
    x = linalg.adjoint_GMRES(lambda v: Ad @ v, lambda v: Ad.T @ v, torch.as_tensor(b, device="cuda"), 140, 130, 16,
                             outer=2, precond_left=[lambda v, mode: dd * v])
    xo, _ = K.adjoint_GMRES(lambda v: A @ v, lambda v: A.T @ v, b, 140, 130, 16, outer=2,
                            precond_left=[lambda v, mode: d * v])
    assert _rel(x, xo) < 1e-10


# --- the MHD objective -------------------------------------------------------

KW = dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=0, rot=False)


def _mhd(n=64):
    u0 = initial_condition(3, n)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **KW)
    pdt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **KW)
    x = {"fields": torch.as_tensor(u0, device="cuda"), "T": 0.1, "sx": 0.35}
    f_t = lambda d: O.objective_RPO(d, pdt, "Lawson_RK4", xp=O.TORCH)
    prim = {"fields": torch.from_numpy(u0), "T": torch.tensor(0.1, dtype=torch.float64),
            "sx": torch.tensor(0.35, dtype=torch.float64)}
    return u0, pd, x, f_t, prim


def _oracle_flat(f_t, prim, n):
    def A(v):
        t = O.unravel_dict(torch.from_numpy(np.ascontiguousarray(v)), n)
        t = {"fields": t["fields"], "T": t["T"], "sx": t["sx"]}        # the primal's key order
        return O.ravel_dict(tjvp(f_t, (prim,), (t,))[1], xp=O.TORCH).detach().numpy()

    def f_vec(v):
        d = O.unravel_dict(torch.from_numpy(np.ascontiguousarray(v)), n)
        return O.ravel_dict(f_t(d), xp=O.TORCH).detach().numpy()
    return A, f_vec


@pytest.mark.parametrize("s0", [1e3, 0.05])
def test_hookstep_v2_mhd_matches_oracle(cuda, s0):
    n = 64
    u0, pd, x, f_t, prim = _mhd(n)
    obj = E.Objective(pd, "Lawson_RK4")

    def A(v):
        t = unflatten(v, n)
        return flatten(obj.jvp(x, {"fields": t["fields"].contiguous(), "T": t["T"], "sx": t["sx"]}))

    b = flatten(obj(x))
    new, s, rr = linalg.newton_gmres_hookstep_v2(A, b, 5, s0, obj, x)
    Ao, fo = _oracle_flat(f_t, prim, n)
    x0 = O.ravel_dict({"fields": u0, "T": 0.1, "sx": 0.35})
    xo, so, rro = K.newton_gmres_hookstep_v2(Ao, fo(x0), 5, s0, fo, x0)
    assert _rel(flatten(new), xo) < 1e-8 and s == so
    assert abs(float(rr) - rro) <= 1e-6 * rro


def test_diagonal_estimates_mhd_match_oracle(cuda):
    n = 64
    u0, pd, x, f_t, prim = _mhd(n)
    obj = E.Objective(pd, "Lawson_RK4")
    Ao, _ = _oracle_flat(f_t, prim, n)
    lin_fields = lambda zp: np.stack([Ao(r)[1:-1] for r in zp])
    ds = preconditioners.diagonal_estimate_spatial(x, obj.jvp, k=2, batch=4, seed=0)
    dso = K.diagonal_estimate_spatial(lin_fields, 2 * n * n, k=2, batch=4, seed=0)
    assert _rel(ds.reshape(-1), dso) < 1e-11
    df = preconditioners.diagonal_estimate_fourier(x, obj.jvp, k=2, batch=4, seed=0)
    dfo = K.diagonal_estimate_fourier(lin_fields, (2, n, n), k=2, batch=4, seed=0)
    assert _rel(df, dfo) < 1e-11
    M = preconditioners.diagonal_preconditioner_spatial(x, pd, obj.jvp, k=2, batch=4, seed=0)
    v = flatten(x)
    mv = M(v, "no_trans")
    assert float(mv[0]) == float(v[0]) and torch.allclose(mv[1:-1], v[1:-1] / ds.reshape(-1))


def _perturbed_rpo6(eps):
    d = np.load("tests/golden/solution_Re40_RPO6.npz")
    n = d["fields"].shape[-1]
    pd = E.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=d["b0"], forcing="kolmogorov",
                           num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
                           shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))
    u = torch.as_tensor(d["fields"] + eps * initial_condition(99, n, amp=1.0), device="cuda")
    return {"fields": E.dealias(u, pd), "T": float(d["T"]) * (1 + eps), "sx": float(d["sx"])}, pd


def test_newton_hookstep_iteration_converges(cuda):
    """newton_hookstep_v2.py's loop on the reference's RPO6 perturbed off the
    orbit (16 Krylov vectors of J itself): every iteration lowers the
    residual, two of them by more than 10x, and the accepted steps double s."""
    x, pd = _perturbed_rpo6(1e-3)
    fs = [float(torch.linalg.norm(E.objective_RPO(x, pd, "Lawson_RK4")["fields"]))]
    s = 100.0
    for _ in range(2):
        x, s, st = drivers.newton_hookstep_iteration(x, pd, "Lawson_RK4", inner=16, s=s)
        fs.append(float(torch.linalg.norm(E.objective_RPO(x, pd, "Lawson_RK4")["fields"])))
    assert fs[2] < fs[1] < fs[0] and fs[2] < 0.1 * fs[0], (fs, st)
    assert s == 400.0


def test_newton_block_gmres_converges(cuda):
    """A Newton step solved by block GMRES over batched JVPs (8 tangents per
    product, 4 products) shrinks the residual of the perturbed RPO6."""
    x, pd = _perturbed_rpo6(1e-3)
    f0 = float(torch.linalg.norm(E.objective_RPO(x, pd, "Lawson_RK4")["fields"]))
    new, st = drivers.newton_block_gmres_update(x, pd, "Lawson_RK4", block=8, m=4)
    f1 = float(torch.linalg.norm(E.objective_RPO(new, pd, "Lawson_RK4")["fields"]))
    assert f1 < f0, (f0, f1, st)
