"""JVP and VJP of objective_RPO in the classic RK4 and Lawson-RK6 modes
(mismatch_RPO, jax_scripts/lib/loss_functions.py:49-56 and :66-71; the steppers
of jax_scripts/lib/timestepping.py:17-44 and :83-125) against torch.func.jvp /
torch.func.vjp of the oracle's torch restatement, as jax.jvp / jax.vjp of the
reference give them; plus the dot-product test <u, J v> = <J^T u, v>.

Tolerances: 1e-12 relative L2 on the fields (FP64), 1e-12 relative on the
phase-condition and T / sx components; adjointness 1e-12.  RK4 carries the
modes outside the box unchanged, so it is also checked on a state with energy
outside the box."""
import numpy as np
import pytest
import torch
from torch.func import jvp as tjvp, vjp as tvjp

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200.synthetic import initial_condition
from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12

CASES = [   # (mode, n, param kwargs, T, dealiased input)
    ("RK4", 64, dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=0, rot=False), 0.1, True),
    ("RK4", 64, dict(num_checkpoints=1, ministeps=12, shift_reflect_ny=3, rot=True), 0.08, False),
    ("Lawson_RK6", 64, dict(steps=24, shift_reflect_ny=1, rot=False), 0.2, True),
    ("Lawson_RK6", 64, dict(steps=16, shift_reflect_ny=6, rot=True), 0.15, False),
    ("RK4", 128, dict(num_checkpoints=2, ministeps=6, shift_reflect_ny=2, rot=False), 0.03, True),
    # 128^2: 24 steps over T=0.1 (h ~ 0.004); at h ~ 0.008 the explicit stages amplify rounding at
    # k_max = 42 (the oracle's own numpy and torch forms then differ by 6e-10 after 12 steps)
    ("Lawson_RK6", 128, dict(steps=24, shift_reflect_ny=0, rot=True), 0.1, True),
]


def _u0(n, dealiased):
    u = initial_condition(5, n)
    if not dealiased:   # energy outside the box (RK4 carries it, Lawson-RK6 zeroes it)
        u = u + 0.05 * np.random.default_rng(1).standard_normal(u.shape)
    return u


def _t(x):
    return torch.tensor(x, dtype=torch.float64)


def _setup(mode, n, kw, T, dealiased):
    u0 = _u0(n, dealiased)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    pdt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **kw)
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": 0.35}
    prim_t = {"fields": torch.from_numpy(u0), "T": _t(T), "sx": _t(0.35)}
    f = lambda d: O.objective_RPO(d, pdt, mode, xp=O.TORCH)
    return u0, pd, prim, prim_t, f


@pytest.mark.parametrize("mode,n,kw,T,dealiased", CASES)
def test_jvp_matches_oracle(cuda, mode, n, kw, T, dealiased):
    u0, pd, prim, prim_t, f = _setup(mode, n, kw, T, dealiased)
    rng = np.random.default_rng(11)
    du = np.stack([initial_condition(20 + i, n) * 0.1 + 0.01 * rng.standard_normal((2, n, n)) for i in range(3)])
    dT, dsx = np.array([0.0, 0.3, -1.2]), np.array([0.0, -0.5, 0.8])
    obj = E.Objective(pd, mode)
    val, got = obj.linearize_jvp(prim, {"fields": torch.as_tensor(du, device="cuda"), "T": _t(dT), "sx": _t(dsx)})
    want_val = O.objective_RPO({"fields": u0, "T": T, "sx": 0.35},
                               O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw), mode)
    assert rel_l2(val["fields"].cpu().numpy(), want_val["fields"]) < TOL
    for b in range(3):
        _, want = tjvp(f, (prim_t,), ({"fields": torch.from_numpy(du[b]), "T": _t(dT[b]), "sx": _t(dsx[b])},))
        assert rel_l2(got["fields"][b].cpu().numpy(), want["fields"].detach().numpy()) < TOL, b
        for k in ("T", "sx"):
            w = float(want[k])
            assert abs(float(got[k][b]) - w) <= TOL * max(abs(w), 1e-30) + 1e-18, (k, b)


@pytest.mark.parametrize("mode,n,kw,T,dealiased", CASES)
def test_vjp_matches_oracle(cuda, mode, n, kw, T, dealiased):
    u0, pd, prim, prim_t, f = _setup(mode, n, kw, T, dealiased)
    rng = np.random.default_rng(5)
    cf = np.stack([rng.standard_normal((2, n, n)) for _ in range(2)])
    cT, csx = np.array([0.7, -0.2]), np.array([0.0, 1.3])
    obj = E.Objective(pd, mode)
    _, jacT = E.vjp(obj, prim)
    got = jacT({"fields": torch.as_tensor(cf, device="cuda"), "T": _t(cT), "sx": _t(csx)})[0]
    _, fn = tvjp(f, prim_t)
    for b in range(2):
        want = fn({"fields": torch.from_numpy(cf[b]), "T": _t(cT[b]), "sx": _t(csx[b])})[0]
        assert rel_l2(got["fields"][b].cpu().numpy(), want["fields"].detach().numpy()) < TOL, b
        for k in ("T", "sx"):
            w = float(want[k])
            assert abs(float(got[k][b]) - w) <= TOL * max(abs(w), 1.0), (k, b)


@pytest.mark.parametrize("mode", ["RK4", "Lawson_RK6"])
def test_dot_product_adjointness(cuda, mode):
    """(u, J v) == (J^T u, v) (timestepping.py:496-504's check) at 64^2."""
    n = 64
    kw = CASES[0][2] if mode == "RK4" else CASES[2][2]
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    obj = E.Objective(pd, mode)
    prim = {"fields": torch.as_tensor(initial_condition(6, n), device="cuda"), "T": 0.1, "sx": -0.4}
    rng = np.random.default_rng(8)
    v = {"fields": torch.as_tensor(rng.standard_normal((2, n, n)), device="cuda"), "T": 0.3, "sx": -0.7}
    u = {"fields": torch.as_tensor(rng.standard_normal((2, n, n)), device="cuda"), "T": 1.1, "sx": 0.4}
    Jv = obj.jvp(prim, v)
    _, jacT = E.vjp(obj, prim)
    JTu = jacT(u)[0]
    lhs = float(torch.sum(u["fields"] * Jv["fields"])) + 1.1 * float(Jv["T"]) + 0.4 * float(Jv["sx"])
    rhs = float(torch.sum(JTu["fields"] * v["fields"])) + 0.3 * float(JTu["T"]) - 0.7 * float(JTu["sx"])
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))
