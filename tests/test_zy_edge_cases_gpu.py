"""Edge cases of the device path: empty batches return empty results without a
launch, a tangent batch of one precision pushed through a primal of the
other is converted to the primal's precision, and grid sizes or modes that
the library does not provide end in an error status, not a launch.  The
non-empty results are compared with the same calls on well-formed inputs.
This file sorts after the parity tests so that a run stopping at the first
failure has run those first."""
import numpy as np
import pytest
import torch

import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import _lib, autodiff, linalg
from ecs_mhd_2d_b200.synthetic import initial_condition

pytestmark = pytest.mark.gpu

KW = dict(num_checkpoints=1, ministeps=8, shift_reflect_ny=1, rot=False)


@pytest.fixture(scope="module")
def setup(cuda):
    n = 64
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **KW)
    x = {"fields": torch.as_tensor(initial_condition(0, n), device="cuda"), "T": 0.05, "sx": 0.2}
    return n, pd, x


def _launches(ctx):
    return ctx.lib.ecs_launch_count(ctx.handle)


def _rel(a, b):
    return float(torch.linalg.norm(a - b) / max(float(torch.linalg.norm(b)), 1e-300))


def test_empty_batches(setup):
    n, pd, x = setup
    empty = {"fields": torch.zeros(0, 2, n, n, dtype=torch.float64, device="cuda"),
             "T": torch.zeros(0), "sx": torch.zeros(0)}
    out = E.objective_RPO(empty, pd, "Lawson_RK4")
    assert out["fields"].shape == (0, 2, n, n) and out["T"].shape == (0,) and out["sx"].shape == (0,)
    loss, infos = E.loss_RPO(empty, pd, "Lawson_RK4")
    assert loss.shape == (0,) and infos == []
    assert E.dealias(empty["fields"], pd).shape == (0, 2, n, n)
    fh = torch.zeros(0, 2, n, n // 2 + 1, dtype=torch.complex128, device="cuda")
    assert E.state_vel(fh, pd, False).shape == fh.shape
    assert E.lawson_rk4(fh, 0.1, 2, pd).shape == fh.shape
    assert E.integrate(fh, 0.1, 2, pd, "TDRK4").shape == fh.shape
    obj = autodiff.Objective(pd, "Lawson_RK4")
    d = obj.jvp(x, empty)
    assert d["fields"].shape == (0, 2, n, n) and d["T"].shape == (0,)
    g = autodiff._vjp_call(obj, x, empty)
    assert g["fields"].shape == (0, 2, n, n)
    # the primal value still comes back with an empty tangent batch
    val, tan = obj.linearize_jvp(x, empty)
    ref = E.objective_RPO(x, pd, "Lawson_RK4")
    assert _rel(val["fields"], ref["fields"]) < 1e-12 and tan["fields"].shape == (0, 2, n, n)


def test_tangent_precision_follows_the_primal(setup):
    n, pd, x = setup
    obj = autodiff.Objective(pd, "Lawson_RK4")
    rng = np.random.default_rng(3)
    t32 = torch.as_tensor(rng.standard_normal((3, 2, n, n)), dtype=torch.float32, device="cuda")
    tan32 = {"fields": t32, "T": torch.zeros(3), "sx": torch.zeros(3)}
    tan64 = {"fields": t32.double(), "T": torch.zeros(3), "sx": torch.zeros(3)}
    a, b = obj.jvp(x, tan32), obj.jvp(x, tan64)
    assert a["fields"].dtype == torch.float64
    assert _rel(a["fields"], b["fields"]) < 1e-13 and _rel(a["T"], b["T"]) < 1e-12
    ga, gb = autodiff._vjp_call(obj, x, tan32), autodiff._vjp_call(obj, x, tan64)
    assert ga["fields"].dtype == torch.float64 and _rel(ga["fields"], gb["fields"]) < 1e-13


def test_mismatched_tangent_grid_never_launches(setup):
    n, pd, x = setup
    obj = autodiff.Objective(pd, "Lawson_RK4")
    obj.linearize(x, batch=2)
    before = _launches(obj._ctx)
    big = {"fields": torch.zeros(2, 2, 2 * n, 2 * n, dtype=torch.float64, device="cuda"),
           "T": torch.zeros(2), "sx": torch.zeros(2)}
    with pytest.raises(ValueError, match="grid side"):
        obj.jvp(x, big)
    with pytest.raises(ValueError, match="grid side"):
        obj.linearize_jvp(x, big)
    with pytest.raises(ValueError, match="grid side"):
        autodiff._vjp_call(obj, x, big)
    assert _launches(obj._ctx) == before


def test_unsupported_grid_and_mode_are_status_errors(setup):
    n, pd, x = setup
    pd96 = E.make_param_dict(96, 1 / 40, 1 / 40, forcing="kolmogorov+", **KW)
    x96 = {"fields": torch.zeros(2, 96, 96, dtype=torch.float64, device="cuda"), "T": 0.05, "sx": 0.0}
    with pytest.raises(_lib.EcsError) as ei:
        E.objective_RPO(x96, pd96, "Lawson_RK4")
    assert ei.value.code == 6                         # ECS_ERR_UNSUPPORTED
    obj = autodiff.Objective(pd, "Lawson_RK4")
    obj.cfg.mode = 42                                 # a mode code the library does not know
    with pytest.raises(_lib.EcsError) as ei:
        obj.linearize(x)
    assert ei.value.code == 3                         # ECS_ERR_BAD_MODE


def test_krylov_vector_of_wrong_length(cuda):
    b = torch.ones(64, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="length 64"):
        linalg.gmres(lambda v: v[:32], b, 4)
