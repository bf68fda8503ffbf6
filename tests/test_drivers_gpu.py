"""Newton-GMRES and adjoint-descent iterations (jax_scripts/newton.py:151-215,
jax_scripts/adjoint_descent.py:93-114) on a reference solution perturbed off
the orbit: a Newton step must shrink the residual sharply, adjoint descent
must lower the loss."""
import numpy as np
import pytest
import torch

import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import drivers
from ecs_mhd_2d_b200.synthetic import initial_condition

pytestmark = pytest.mark.gpu


def perturbed_rpo6(eps):
    d = np.load("tests/golden/solution_Re40_RPO6.npz")
    n = d["fields"].shape[-1]
    pd = E.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=d["b0"], forcing="kolmogorov",
                           num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
                           shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))
    pert = eps * initial_condition(99, n, amp=1.0)
    u = torch.as_tensor(d["fields"] + pert, device="cuda")
    u = E.dealias(u, pd)
    return {"fields": u, "T": float(d["T"]) * (1 + eps), "sx": float(d["sx"])}, pd


def test_newton_gmres_step_converges(cuda):
    x, pd = perturbed_rpo6(1e-3)
    f0 = float(torch.linalg.norm(E.objective_RPO(x, pd, "Lawson_RK4")["fields"]))
    new, st = drivers.newton_gmres_update(x, pd, "Lawson_RK4", inner=16, use_transpose=True)
    f1 = float(torch.linalg.norm(E.objective_RPO(new, pd, "Lawson_RK4")["fields"]))
    assert st["damp"] == 1.0
    assert f1 < 0.05 * f0, (f0, f1, st)


def test_adjoint_descent_lowers_loss(cuda):
    x, pd = perturbed_rpo6(1e-2)
    m, v = {}, {}
    losses = []
    for t in range(1, 4):
        x, m, v, loss, info = drivers.adjoint_descent_step(x, pd, "Lawson_RK4", m, v, t, lr=1e-3)
        losses.append(loss)
    assert losses[-1] < losses[0]


def test_mixed_precision_newton_reaches_fp64_accuracy(cuda):
    """FP32 Jacobian products with FP64 residuals converge (inexact Newton,
    linearly); one FP64 refinement sweep then reaches FP64-level closure."""
    x, pd = perturbed_rpo6(1e-4)
    new, hist = drivers.mixed_precision_newton(x, pd, "Lawson_RK4", iters=2, inner=16, refine=1)
    fp32 = [h for h in hist if h.get("jacobian") == "fp32"]
    assert fp32[-1]["rel_err"] < fp32[0]["rel_err"] or hist[-2]["rel_err"] < fp32[0]["rel_err"], hist
    assert hist[-1]["final_rel_err"] < 1e-8, hist
