"""The other shooting modes of mismatch_RPO (loss_functions.py:48-85) on the
CUDA path against the oracle: classic RK4 (dissipation in the right-hand side),
Lawson_RK6 and TDRK4 (two-derivative RK4, whose stage Jacobian-vector products
run through the tangent row pass).  Tolerance 1e-12 relative L2 (FP64), as for
the Lawson-RK4 objective.  RK4 and TDRK4 carry the modes outside the 2/3 box
unchanged, so non-dealiased inputs are included."""
import numpy as np
import pytest
import torch

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200.synthetic import initial_condition
from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12

CASES = [
    ("RK4", dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=0, rot=False), 0.1),
    ("RK4", dict(num_checkpoints=1, ministeps=20, shift_reflect_ny=3, rot=True), 0.12),
    ("Lawson_RK6", dict(steps=24, shift_reflect_ny=1, rot=False), 0.2),
    ("Lawson_RK6", dict(steps=40, shift_reflect_ny=6, rot=True), 0.3),
    ("TDRK4", dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=0, rot=False), 0.1),
    ("TDRK4", dict(num_checkpoints=3, ministeps=11, shift_reflect_ny=5, rot=True), 0.15),
]


def _u0(n, dealiased):
    u = initial_condition(5, n)
    if not dealiased:   # add energy outside the box (carried unchanged by RK4 / TDRK4)
        rng = np.random.default_rng(1)
        u = u + 0.05 * rng.standard_normal(u.shape)
    return u


@pytest.mark.parametrize("mode,kw,T", CASES)
@pytest.mark.parametrize("dealiased", [True, False])
def test_objective_and_loss_modes(cuda, mode, kw, T, dealiased):
    n = 64
    u0 = _u0(n, dealiased)
    opd = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    inp = {"fields": u0, "T": T, "sx": 0.4}
    dinp = {"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": 0.4}
    want = O.objective_RPO(inp, opd, mode)
    got = E.objective_RPO(dinp, pd, mode)
    assert rel_l2(got["fields"].cpu().numpy(), want["fields"]) < TOL
    wl, _ = O.loss_RPO(inp, opd, mode)
    gl, _ = E.loss_RPO(dinp, pd, mode)
    assert abs(float(gl) - float(wl)) <= TOL * abs(float(wl))


@pytest.mark.parametrize("mode", ["RK4", "Lawson_RK6", "TDRK4"])
def test_modes_batch_equals_single(cuda, mode):
    n = 64
    kw = dict(num_checkpoints=1, ministeps=24, steps=24, shift_reflect_ny=1, rot=False)   # explicit RK4: dt <= 0.008
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    us = np.stack([initial_condition(s, n) for s in range(3)])
    T = torch.tensor([0.1, 0.2, 0.15], dtype=torch.float64)
    sx = torch.tensor([0.0, 0.5, -1.0], dtype=torch.float64)
    batch = E.objective_RPO({"fields": torch.as_tensor(us, device="cuda"), "T": T, "sx": sx}, pd, mode)
    for b in range(3):
        one = E.objective_RPO({"fields": torch.as_tensor(us[b], device="cuda"), "T": float(T[b]),
                               "sx": float(sx[b])}, pd, mode)
        assert torch.equal(one["fields"], batch["fields"][b])


def test_tdrk4_closes_reference_solution(cuda):
    """The reference's Re40/TW1 closes to 4e-15 under the oracle's TDRK4 (and
    only to 1e-9 under Lawson-RK4): the mode it was converged with.  The GPU
    TDRK4 must close it to the 1e-12 budget."""
    d = np.load("tests/golden/solution_Re40_TW1.npz")
    n = d["fields"].shape[-1]
    pd = E.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=d["b0"], forcing="kolmogorov",
                           num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
                           shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))
    out = E.objective_RPO({"fields": torch.as_tensor(d["fields"], device="cuda"), "T": float(d["T"]),
                           "sx": float(d["sx"])}, pd, "TDRK4")
    r = float(torch.linalg.norm(out["fields"]) / np.linalg.norm(d["fields"]))
    assert r < 1e-12, r


@pytest.mark.parametrize("ny,rot,dealiased", [(0, False, True), (3, True, False)])
def test_tdrk4_jvp_matches_oracle(cuda, ny, rot, dealiased):
    """JVP of objective_RPO in TDRK4 mode (the reference Newton driver's default,
    jax_scripts/newton.py:70) against torch.func.jvp of the oracle's torch
    restatement, whose stage Jacobian-vector products are themselves
    torch.func.jvp (forward over forward, as jax.jvp of jax.jvp)."""
    from torch.func import jvp as tjvp
    n, T, sx = 64, 0.1, 0.35
    kw = dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=ny, rot=rot)
    u0 = _u0(n, dealiased)
    rng = np.random.default_rng(11)
    du = np.stack([initial_condition(20 + i, n) * 0.1 + 0.01 * rng.standard_normal((2, n, n)) for i in range(3)])
    dT = np.array([0.0, 0.3, -1.2]); dsx = np.array([0.0, -0.5, 0.8])
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    pdt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **kw)
    obj, jac = E.compile_objective_and_Jacobian({"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": sx},
                                                pd, "TDRK4")
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": sx}
    got = jac(prim, {"fields": torch.as_tensor(du, device="cuda"), "T": torch.tensor(dT), "sx": torch.tensor(dsx)})
    f = lambda d: O.objective_RPO(d, pdt, "TDRK4", xp=O.TORCH)
    for b in range(3):
        p_t = {"fields": torch.from_numpy(u0), "T": torch.tensor(T, dtype=torch.float64),
               "sx": torch.tensor(sx, dtype=torch.float64)}
        t_t = {"fields": torch.from_numpy(du[b]), "T": torch.tensor(dT[b], dtype=torch.float64),
               "sx": torch.tensor(dsx[b], dtype=torch.float64)}
        _, want = tjvp(f, (p_t,), (t_t,))
        assert rel_l2(got["fields"][b].cpu().numpy(), want["fields"].detach().numpy()) < TOL, b
        for k in ("T", "sx"):
            w = float(want[k])
            assert abs(float(got[k][b]) - w) <= TOL * max(abs(w), 1e-30) + 1e-18


@pytest.mark.parametrize("ny,rot,dealiased", [(1, False, True), (4, True, False)])
def test_tdrk4_vjp_matches_oracle(cuda, ny, rot, dealiased):
    """VJP of objective_RPO in TDRK4 mode (jax.vjp(obj, input_dict), the
    transpose preconditioner of jax_scripts/newton.py:168-169) against
    torch.func.vjp of the oracle's torch restatement (reverse over forward)."""
    from torch.func import vjp as tvjp
    n, T, sx = 64, 0.1, 0.35
    kw = dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=ny, rot=rot)
    u0 = _u0(n, dealiased)
    rng = np.random.default_rng(12)
    cf = rng.standard_normal((2, n, n))
    cT, csx = 0.7, -0.4
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    pdt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **kw)
    obj = E.Objective(pd, "TDRK4")
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": sx}
    _, jacT = E.vjp(obj, prim)
    got = jacT({"fields": torch.as_tensor(cf, device="cuda"), "T": cT, "sx": csx})[0]
    f = lambda d: O.objective_RPO(d, pdt, "TDRK4", xp=O.TORCH)
    p_t = {"fields": torch.from_numpy(u0), "T": torch.tensor(T, dtype=torch.float64),
           "sx": torch.tensor(sx, dtype=torch.float64)}
    _, pull = tvjp(f, p_t)
    (want,) = pull({"fields": torch.from_numpy(cf), "T": torch.tensor(cT, dtype=torch.float64),
                    "sx": torch.tensor(csx, dtype=torch.float64)})
    assert rel_l2(got["fields"].cpu().numpy(), want["fields"].detach().numpy()) < TOL
    # the T cotangent is a sum over steps of four inner products <xbar, x>/h, each much
    # larger than the sum; both sides accumulate them in different orders (measured
    # 3.6e-12 relative), so the scalars get 1e-10
    for k in ("T", "sx"):
        w = float(want[k])
        assert abs(float(got[k]) - w) <= 1e-10 * max(abs(w), 1e-30) + 1e-18, (k, float(got[k]), w)


def test_tdrk4_dot_product_adjointness(cuda):
    """<J v, u> = <v, J^T u> for the TDRK4 objective (timestepping.py:496-504's check)."""
    n = 64
    kw = dict(num_checkpoints=1, ministeps=12, shift_reflect_ny=2, rot=True)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    u0 = _u0(n, False)
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": 0.08, "sx": 0.2}
    rng = np.random.default_rng(3)
    v = {"fields": torch.as_tensor(rng.standard_normal((2, n, n)), device="cuda"), "T": 0.3, "sx": -0.6}
    u = {"fields": torch.as_tensor(rng.standard_normal((2, n, n)), device="cuda"), "T": -0.2, "sx": 0.9}
    obj = E.Objective(pd, "TDRK4")
    jv = obj.jvp(prim, v)
    _, jacT = E.vjp(obj, prim)
    ju = jacT(u)[0]
    lhs = float((jv["fields"] * u["fields"]).sum()) + float(jv["T"]) * u["T"] + float(jv["sx"]) * u["sx"]
    rhs = float((v["fields"] * ju["fields"]).sum()) + v["T"] * float(ju["T"]) + v["sx"] * float(ju["sx"])
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), abs(rhs))
