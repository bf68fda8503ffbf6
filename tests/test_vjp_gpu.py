"""VJP / adjoint gradient of the CUDA path: against torch.func.vjp of the oracle's
torch twin (1e-12 relative), the dot-product test <u, J v> = <J^T u, v> between the
CUDA JVP and VJP (1e-12), and central finite differences of the loss (1e-6, the FD
truncation level)."""
import numpy as np
import pytest
import torch
from torch.func import vjp as tvjp

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200.synthetic import initial_condition
from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12
TOL_43 = 1e-10   # adaptive step-size controller sensitivity, see test_parity_gpu.TOL_43

CASES = [
    ("Lawson_RK4", dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=0, rot=False)),
    ("Lawson_RK4", dict(num_checkpoints=1, ministeps=12, shift_reflect_ny=3, rot=True)),
    ("Lawson_RK43", dict(shift_reflect_ny=2, rot=False, adaptive_dict={"atol": 1e-5, "checkpoints": 4, "max_steps_per_checkpoint": 16})),
    ("Lawson_RK43", dict(shift_reflect_ny=1, rot=True, adaptive_dict={"atol": 1e-7, "checkpoints": 4, "max_steps_per_checkpoint": 32})),
]


def oracle_vjp(u0, T, sx, cot, pd_t, mode):
    f = lambda d: O.objective_RPO(d, pd_t, mode, xp=O.TORCH)
    prim = {"fields": torch.from_numpy(u0), "T": torch.tensor(T, dtype=torch.float64),
            "sx": torch.tensor(sx, dtype=torch.float64)}
    _, fn = tvjp(f, prim)
    c = {"fields": torch.from_numpy(cot[0]), "T": torch.tensor(cot[1], dtype=torch.float64),
         "sx": torch.tensor(cot[2], dtype=torch.float64)}
    return {k: v.detach().numpy() for k, v in fn(c)[0].items()}


@pytest.mark.parametrize("mode,kw", CASES)
def test_vjp_matches_oracle(cuda, mode, kw):
    n, T, sx = 64, 0.1, 0.35
    u0 = initial_condition(3, n)
    rng = np.random.default_rng(5)
    cf = np.stack([rng.standard_normal((2, n, n)) for _ in range(2)])
    cT = np.array([0.7, -0.2]); csx = np.array([0.0, 1.3])
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    pdt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **kw)
    obj = E.Objective(pd, mode)
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": sx}
    out, jacT = E.vjp(obj, prim)
    got = jacT({"fields": torch.as_tensor(cf, device="cuda"), "T": torch.tensor(cT), "sx": torch.tensor(csx)})[0]
    for b in range(2):
        want = oracle_vjp(u0, T, sx, (cf[b], cT[b], csx[b]), pdt, mode)
        tol = TOL_43 if mode == "Lawson_RK43" else TOL
        assert rel_l2(got["fields"][b].cpu().numpy(), want["fields"]) < tol, b
        for k in ("T", "sx"):
            assert abs(float(got[k][b]) - float(want[k])) <= tol * max(abs(float(want[k])), 1.0), (k, b)


@pytest.mark.parametrize("mode,kw", CASES)
def test_dot_product_adjointness(cuda, mode, kw):
    """(u, J v) == (J^T u, v), the reference's own check (timestepping.py:496-504)."""
    n = 64
    u0 = initial_condition(6, n)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    obj = E.Objective(pd, mode)
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": 0.12, "sx": -0.4}
    rng = np.random.default_rng(8)
    v = {"fields": torch.as_tensor(rng.standard_normal((2, n, n)), device="cuda"), "T": 0.3, "sx": -0.7}
    u = {"fields": torch.as_tensor(rng.standard_normal((2, n, n)), device="cuda"), "T": 1.1, "sx": 0.4}
    Jv = obj.jvp(prim, v)
    _, jacT = E.vjp(obj, prim)
    JTu = jacT(u)[0]
    lhs = float(torch.sum(u["fields"] * Jv["fields"])) + 1.1 * float(Jv["T"]) + 0.4 * float(Jv["sx"])
    rhs = float(torch.sum(JTu["fields"] * v["fields"])) + 0.3 * float(JTu["T"]) - 0.7 * float(JTu["sx"])
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))


def test_loss_gradient_finite_differences(cuda):
    n = 64
    u0 = initial_condition(1, n)
    kw = dict(num_checkpoints=2, ministeps=16, shift_reflect_ny=1, rot=False)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    inp = {"fields": torch.as_tensor(u0, device="cuda"), "T": 0.3, "sx": 0.2}
    (loss, _), g = E.loss_and_grad(inp, pd, "Lawson_RK4")
    rng = np.random.default_rng(2)
    d = torch.as_tensor(rng.standard_normal((2, n, n)), device="cuda")
    dT, dsx, eps = 0.5, -0.3, 1e-6
    lp, _ = E.loss_RPO({"fields": inp["fields"] + eps * d, "T": 0.3 + eps * dT, "sx": 0.2 + eps * dsx}, pd, "Lawson_RK4")
    lm, _ = E.loss_RPO({"fields": inp["fields"] - eps * d, "T": 0.3 - eps * dT, "sx": 0.2 - eps * dsx}, pd, "Lawson_RK4")
    fd = (float(lp) - float(lm)) / (2 * eps)
    an = float(torch.sum(g["fields"] * d)) + dT * float(g["T"]) + dsx * float(g["sx"])
    assert abs(fd - an) <= 1e-6 * abs(an)


def test_autograd_function(cuda):
    n = 64
    u0 = torch.as_tensor(initial_condition(2, n), device="cuda").requires_grad_(True)
    T = torch.tensor(0.2, dtype=torch.float64, device="cuda", requires_grad=True)
    sx = torch.tensor(0.1, dtype=torch.float64, device="cuda", requires_grad=True)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", num_checkpoints=1, ministeps=16,
                           shift_reflect_ny=0, rot=False)
    loss = E.loss_rpo_autograd(u0, T, sx, pd, "Lawson_RK4")
    loss.backward()
    (l2, _), g = E.loss_and_grad({"fields": u0.detach(), "T": 0.2, "sx": 0.1}, pd, "Lawson_RK4")
    assert torch.allclose(u0.grad, g["fields"], rtol=0, atol=1e-14 * float(g["fields"].abs().max()))
    assert abs(float(T.grad) - float(g["T"])) <= 1e-12 * abs(float(g["T"]))


def test_autograd_forward_and_backward_split(cuda):
    """The adjoint sweep runs in backward only (as jax.value_and_grad splits it,
    jax_scripts/adjoint_descent.py:91): under torch.no_grad the op launches
    exactly what the plain loss_RPO launches; with grad enabled backward adds
    the adjoint launches; the upstream gradient scales the result; the
    normalised loss matches loss_and_grad(normalized=True)."""
    from ecs_mhd_2d_b200 import context
    n = 64
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", num_checkpoints=2, ministeps=8,
                           shift_reflect_ny=1, rot=False, ckpt_every=4)
    u0h = initial_condition(9, n)
    inp = {"fields": torch.as_tensor(u0h, device="cuda"), "T": 0.15, "sx": 0.3}
    ctx = context.get_context(pd, n, torch.float64, 1)
    count = lambda: (torch.cuda.synchronize(), ctx.lib.ecs_launch_count(ctx.handle))[1]

    c0 = count()
    lp, _ = E.loss_RPO(inp, pd, "Lawson_RK4")
    plain = count() - c0
    u0 = torch.as_tensor(u0h, device="cuda").requires_grad_(True)
    T = torch.tensor(0.15, dtype=torch.float64, device="cuda", requires_grad=True)
    sx = torch.tensor(0.3, dtype=torch.float64, device="cuda", requires_grad=True)
    with torch.no_grad():
        c0 = count()
        ln = E.loss_rpo_autograd(u0, T, sx, pd, "Lawson_RK4")
        assert count() - c0 == plain
    assert float(ln) == pytest.approx(float(lp), rel=1e-14)

    c0 = count()
    loss = E.loss_rpo_autograd(u0, T, sx, pd, "Lawson_RK4")
    c1 = count()
    (3.0 * loss).backward()
    assert count() > c1
    assert float(loss) == pytest.approx(float(lp), rel=1e-14)
    (l2, _), g = E.loss_and_grad({"fields": u0.detach(), "T": 0.15, "sx": 0.3}, pd, "Lawson_RK4")
    assert torch.allclose(u0.grad, 3.0 * g["fields"], rtol=1e-13, atol=1e-14 * float(g["fields"].abs().max()))
    assert float(T.grad) == pytest.approx(3.0 * float(g["T"]), rel=1e-12)
    assert float(sx.grad) == pytest.approx(3.0 * float(g["sx"]), rel=1e-12, abs=1e-14)

    u0.grad = T.grad = sx.grad = None
    lossn = E.loss_rpo_autograd(u0, T, sx, pd, "Lawson_RK4", normalized=True)
    lossn.backward()
    (ln2, _), gn = E.loss_and_grad({"fields": u0.detach(), "T": 0.15, "sx": 0.3}, pd, "Lawson_RK4", normalized=True)
    assert float(lossn) == pytest.approx(float(ln2), rel=1e-13)
    assert torch.allclose(u0.grad, gn["fields"], rtol=1e-12, atol=1e-14 * float(gn["fields"].abs().max()))
    assert float(T.grad) == pytest.approx(float(gn["T"]), rel=1e-12)


def test_shared_context_linearisations_do_not_mix(cuda):
    """Two Objectives on the same cached context: a linearisation made by one
    replaces the other's trajectory record, so the other must re-linearise
    before its next JVP instead of reusing the record."""
    n = 64
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", num_checkpoints=1, ministeps=8,
                           shift_reflect_ny=0, rot=False)
    a, b = E.Objective(pd, "Lawson_RK4"), E.Objective(pd, "Lawson_RK4")
    pa = {"fields": torch.as_tensor(initial_condition(1, n), device="cuda"), "T": 0.05, "sx": 0.0}
    pb = {"fields": torch.as_tensor(initial_condition(2, n), device="cuda"), "T": 0.07, "sx": 0.1}
    v = {"fields": torch.as_tensor(initial_condition(3, n), device="cuda"), "T": 0.1, "sx": 0.2}
    ja = a.jvp(pa, v)["fields"].clone()
    b.jvp(pb, v)
    assert torch.equal(a.jvp(pa, v)["fields"], ja)


def test_checkpointed_linearisation_matches_full_record(cuda):
    """Keeping every 5th state and recomputing segments (jax.checkpoint per
    segment, loss_functions.py:63) gives the same JVP and VJP as the full record."""
    n = 64
    u0 = initial_condition(4, n)
    rng = np.random.default_rng(3)
    base = dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=1, rot=True)
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": 0.1, "sx": 0.3}
    v = {"fields": torch.as_tensor(rng.standard_normal((2, n, n)), device="cuda"), "T": 0.2, "sx": -0.1}
    u = {"fields": torch.as_tensor(rng.standard_normal((2, n, n)), device="cuda"), "T": 0.5, "sx": 0.7}
    outs = []
    for ck in (0, 5):
        pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", ckpt_every=ck, **base)
        obj = E.Objective(pd, "Lawson_RK4")
        jv = obj.jvp(prim, v)
        _, jacT = E.vjp(obj, prim)
        outs.append((jv, jacT(u)[0]))
    (j0, g0), (j1, g1) = outs
    assert rel_l2(j1["fields"].cpu().numpy(), j0["fields"].cpu().numpy()) < 1e-14
    assert rel_l2(g1["fields"].cpu().numpy(), g0["fields"].cpu().numpy()) < 1e-14
    assert abs(float(g1["T"]) - float(g0["T"])) <= 1e-13 * abs(float(g0["T"]))
    assert abs(float(g1["sx"]) - float(g0["sx"])) <= 1e-13 * max(abs(float(g0["sx"])), 1.0)


def test_vjp_after_context_growth(cuda):
    """A linearisation at batch 1 followed by a batch of cotangents grows (re-creates)
    the context, which drops the linearisation: the Objective must notice and
    linearise again, even when the new native context reuses the old address."""
    from ecs_mhd_2d_b200 import context
    context.clear_cache()
    n = 64
    kw = CASES[0][1]
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    obj = E.Objective(pd, "Lawson_RK4")
    prim = {"fields": torch.as_tensor(initial_condition(3, n), device="cuda"), "T": 0.1, "sx": 0.35}
    _, jacT = E.vjp(obj, prim)
    rng = np.random.default_rng(6)
    cot = {"fields": torch.as_tensor(rng.standard_normal((3, 2, n, n)), device="cuda"),
           "T": torch.zeros(3, dtype=torch.float64), "sx": torch.zeros(3, dtype=torch.float64)}
    g = jacT(cot)[0]
    g1 = jacT({"fields": cot["fields"][1].contiguous(), "T": 0.0, "sx": 0.0})[0]
    assert torch.isfinite(g["fields"]).all()
    assert torch.allclose(g["fields"][1], g1["fields"], rtol=1e-13, atol=0)
    context.clear_cache()
