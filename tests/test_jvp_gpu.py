"""JVP (Newton-GMRES matvec) of the CUDA path against torch.func.jvp of the oracle's torch twin.

Tolerance: 1e-12 relative L2 on the fields output, 1e-12 relative on the
phase-condition components (FP64)."""
import numpy as np
import pytest
import torch
from torch.func import jvp as tjvp

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200.synthetic import initial_condition
from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12
TOL_43 = 1e-10   # adaptive step-size controller sensitivity, see test_parity_gpu.TOL_43


def oracle_jvp(u0, T, sx, du, dT, dsx, pd_t, mode):
    f = lambda d: O.objective_RPO(d, pd_t, mode, xp=O.TORCH)
    prim = {"fields": torch.from_numpy(u0), "T": torch.tensor(T, dtype=torch.float64),
            "sx": torch.tensor(sx, dtype=torch.float64)}
    tan = {"fields": torch.from_numpy(du), "T": torch.tensor(dT, dtype=torch.float64),
           "sx": torch.tensor(dsx, dtype=torch.float64)}
    _, out = tjvp(f, (prim,), (tan,))
    return {k: v.detach().numpy() for k, v in out.items()}


CASES = [
    ("Lawson_RK4", dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=0, rot=False)),
    ("Lawson_RK4", dict(num_checkpoints=1, ministeps=16, shift_reflect_ny=1, rot=True)),
    ("Lawson_RK43", dict(shift_reflect_ny=2, rot=False, adaptive_dict={"atol": 1e-5, "checkpoints": 4, "max_steps_per_checkpoint": 16})),
    ("Lawson_RK43", dict(shift_reflect_ny=5, rot=True, adaptive_dict={"atol": 1e-7, "checkpoints": 4, "max_steps_per_checkpoint": 32})),
]


@pytest.mark.parametrize("mode,kw", CASES)
def test_jvp_matches_oracle(cuda, mode, kw):
    n, T, sx = 64, 0.1, 0.35
    u0 = initial_condition(3, n)
    rng = np.random.default_rng(11)
    du = np.stack([initial_condition(20 + i, n) * 0.1 + 0.01 * rng.standard_normal((2, n, n)) for i in range(3)])
    dT = np.array([0.0, 0.3, -1.2]); dsx = np.array([0.0, -0.5, 0.8])
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    pdt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **kw)
    obj, jac = E.compile_objective_and_Jacobian({"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": sx}, pd, mode)
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": sx}
    got = jac(prim, {"fields": torch.as_tensor(du, device="cuda"), "T": torch.tensor(dT), "sx": torch.tensor(dsx)})
    for b in range(3):
        want = oracle_jvp(u0, T, sx, du[b], dT[b], dsx[b], pdt, mode)
        tol = TOL_43 if mode == "Lawson_RK43" else TOL
        assert rel_l2(got["fields"][b].cpu().numpy(), want["fields"]) < tol, b
        for k in ("T", "sx"):
            assert abs(float(got[k][b]) - float(want[k])) <= tol * max(abs(float(want[k])), 1e-30) + 1e-18


def test_jvp_linearity_and_batch_consistency(cuda):
    n = 64
    u0 = initial_condition(4, n)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", num_checkpoints=1, ministeps=8,
                           shift_reflect_ny=1, rot=False)
    obj = E.Objective(pd, "Lawson_RK4")
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": 0.05, "sx": 0.1}
    a = torch.as_tensor(initial_condition(7, n), device="cuda")
    b = torch.as_tensor(initial_condition(8, n), device="cuda")
    ja = obj.jvp(prim, {"fields": a, "T": 0.2, "sx": 0.0})
    jb = obj.jvp(prim, {"fields": b, "T": 0.0, "sx": 0.3})
    jab = obj.jvp(prim, {"fields": 2 * a - b, "T": 0.4, "sx": -0.3})
    lin = 2 * ja["fields"] - jb["fields"]
    assert float(torch.linalg.norm(jab["fields"] - lin) / torch.linalg.norm(lin)) < 1e-13
    both = obj.jvp(prim, {"fields": torch.stack([a, b]), "T": torch.tensor([0.2, 0.0], dtype=torch.float64), "sx": torch.tensor([0.0, 0.3], dtype=torch.float64)})
    assert torch.equal(both["fields"][0], ja["fields"]) and torch.equal(both["fields"][1], jb["fields"])


def test_fp32_jvp_against_fp64_oracle(cuda):
    """FP32 stepping and tangent kernels stay within FP32 rounding of the FP64 oracle."""
    n, T, sx = 64, 0.08, 0.2
    kw = dict(num_checkpoints=1, ministeps=16, shift_reflect_ny=1, rot=False)
    u0 = initial_condition(3, n)
    du = initial_condition(21, n) * 0.1
    pd32 = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", data_type=torch.float32, **kw)
    pdt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **kw)
    obj = E.Objective(pd32, "Lawson_RK4")
    prim = {"fields": torch.as_tensor(u0, dtype=torch.float32, device="cuda"), "T": T, "sx": sx}
    got = obj.jvp(prim, {"fields": torch.as_tensor(du, dtype=torch.float32, device="cuda"), "T": 0.3, "sx": -0.4})
    want = oracle_jvp(u0, T, sx, du, 0.3, -0.4, pdt, "Lawson_RK4")
    assert rel_l2(got["fields"].double().cpu().numpy(), want["fields"]) < 5e-5
