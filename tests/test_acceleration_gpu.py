"""Geodesic acceleration (jax_scripts/acceleration.py:103-168) on the device.
The second directional derivative K(v) = d^2 objective[v, v], taken here as a
central difference of two device JVPs, against the exact nested
torch.func.jvp of the oracle (the reference nests jax.jvp), to 2e-6 relative
(the O(eps^2) truncation of the difference is a few 1e-7 at the default eps,
its roundoff ~1e-11); and one accelerated Newton update on the reference's
RPO6 perturbed off the orbit.""" 
import numpy as np
import pytest
import torch
from torch.func import jvp as tjvp

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import drivers
from ecs_mhd_2d_b200.synthetic import initial_condition
from ecs_mhd_2d_b200.utils import flatten

pytestmark = pytest.mark.gpu
KW = dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=0, rot=False)


def test_second_directional_derivative_matches_nested_jvp(cuda):
    n = 64
    u0 = initial_condition(3, n)
    dv = 0.1 * initial_condition(21, n)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **KW)
    pdt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **KW)
    x = {"fields": torch.as_tensor(u0, device="cuda"), "T": 0.1, "sx": 0.35}
    v = flatten({"fields": torch.as_tensor(dv, device="cuda"), "T": 0.3, "sx": -0.2})
    got = drivers.second_directional_derivative(E.Objective(pd, "Lawson_RK4"), x, v).cpu().numpy()
    f = lambda d: O.objective_RPO(d, pdt, "Lawson_RK4", xp=O.TORCH)
    xt = {"fields": torch.from_numpy(u0), "T": torch.tensor(0.1, dtype=torch.float64),
          "sx": torch.tensor(0.35, dtype=torch.float64)}
    vt = {"fields": torch.from_numpy(dv), "T": torch.tensor(0.3, dtype=torch.float64),
          "sx": torch.tensor(-0.2, dtype=torch.float64)}
    want = tjvp(lambda z: tjvp(f, (z,), (vt,))[1], (xt,), (vt,))[1]
    want = O.ravel_dict(want, xp=O.TORCH).detach().numpy()
    assert np.linalg.norm(got - want) <= 2e-6 * np.linalg.norm(want)


def test_geodesic_acceleration_update_converges(cuda):
    d = np.load("tests/golden/solution_Re40_RPO6.npz")
    n = d["fields"].shape[-1]
    pd = E.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=d["b0"], forcing="kolmogorov",
                           num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
                           shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))
    u = torch.as_tensor(d["fields"] + 1e-3 * initial_condition(99, n, amp=1.0), device="cuda")
    x = {"fields": E.dealias(u, pd), "T": float(d["T"]) * (1 + 1e-3), "sx": float(d["sx"])}
    f0 = float(torch.linalg.norm(E.objective_RPO(x, pd, "Lawson_RK4")["fields"]))
    new, st = drivers.geodesic_acceleration_update(x, pd, "Lawson_RK4", inner=16)
    f1 = float(torch.linalg.norm(E.objective_RPO(new, pd, "Lawson_RK4")["fields"]))
    assert f1 < 0.05 * f0, (f0, f1, st)
    assert st["|step2|"] < st["|step1|"]
