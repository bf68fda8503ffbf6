"""Host-side argument checks of the Python layer: a tensor of the wrong shape,
precision or device, a scalar list of the wrong length, an unknown mode or a
forcing of another grid is refused with an exception before any pointer
reaches a kernel (the kernels take their sizes from the context and the call,
so such a tensor would be read past its end).  Every case here raises before
the first device call, so it runs without a GPU."""
import pytest
import torch

import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import autodiff, context as C, linalg, loss_functions, turbulence


@pytest.fixture(scope="module")
def pd64():
    return E.make_param_dict(64, 1 / 40, 1 / 40, forcing="kolmogorov+")


def test_unknown_mode_is_an_error(pd64):
    # loss_functions.py:86-88 prints and exits on an unknown mode
    x = {"fields": torch.zeros(2, 64, 64), "T": 1.0, "sx": 0.0}
    for fn in (E.objective_RPO, E.loss_RPO):
        with pytest.raises(ValueError, match="does not exist"):
            fn(x, pd64, "Lawson_RK5")
    with pytest.raises(ValueError, match="does not exist"):
        autodiff.Objective(pd64, "RK45")
    with pytest.raises(ValueError, match="fixed-step"):
        E.integrate(torch.zeros(2, 64, 33, dtype=torch.complex128), 0.1, 1, pd64, "Lawson_RK43")


@pytest.mark.parametrize("key,val", [("num_checkpoints", 0), ("ministeps", -1), ("ckpt_every", -2),
                                     ("adaptive_dict", {"checkpoints": 0}),
                                     ("adaptive_dict", {"max_steps_per_checkpoint": -4})])
def test_step_counts_checked(key, val):
    pd = E.make_param_dict(64, 1 / 40, 1 / 40, forcing="kolmogorov+", **{key: val})
    with pytest.raises(ValueError, match=">= "):
        E.objective_RPO({"fields": torch.zeros(2, 64, 64), "T": 1.0, "sx": 0.0}, pd,
                        "Lawson_RK43" if key == "adaptive_dict" else "Lawson_RK4")


@pytest.mark.parametrize("shape", [(2, 64, 32), (3, 64, 64), (64, 64), (1, 1, 2, 64, 64), (4, 2, 64, 63)])
def test_fields_shape_checked(pd64, shape):
    x = {"fields": torch.zeros(shape), "T": 1.0, "sx": 0.0}
    with pytest.raises(ValueError, match=r"\[2, n, n\]"):
        E.objective_RPO(x, pd64, "Lawson_RK4")
    with pytest.raises(ValueError, match=r"\[2, n, n\]"):
        E.loss_RPO(x, pd64, "Lawson_RK4")
    with pytest.raises(ValueError, match=r"\[2, n, n\]"):
        loss_functions.dealias(torch.zeros(shape), pd64)


@pytest.mark.parametrize("key", ["T", "sx"])
def test_scalar_count_checked(pd64, key):
    x = {"fields": torch.zeros(3, 2, 64, 64), "T": 1.0, "sx": 0.0}
    x[key] = torch.ones(2)
    with pytest.raises(ValueError, match=f"{key} has 2 values for a batch of 3"):
        E.objective_RPO(x, pd64, "Lawson_RK4")
    x[key] = torch.ones(4)
    with pytest.raises(ValueError, match=f"{key} has 4 values for a batch of 3"):
        E.loss_RPO(x, pd64, "Lawson_RK4")


def test_tangent_and_cotangent_grid_checked_against_the_primal(pd64):
    obj = autodiff.Objective(pd64, "Lawson_RK4")
    primal = {"fields": torch.zeros(2, 64, 64), "T": 1.0, "sx": 0.0}
    tan = {"fields": torch.zeros(4, 2, 128, 128), "T": torch.zeros(4), "sx": torch.zeros(4)}
    with pytest.raises(ValueError, match="tangent fields has grid side 128, the primal has 64"):
        obj.jvp(primal, tan)
    with pytest.raises(ValueError, match="cotangent fields has grid side 128, the primal has 64"):
        autodiff._vjp_call(obj, primal, tan)
    bad = {"fields": torch.zeros(4, 2, 64, 64), "T": torch.zeros(3), "sx": torch.zeros(4)}
    with pytest.raises(ValueError, match="T has 3 values for a batch of 4"):
        obj.jvp(primal, bad)


def test_spectral_inputs_checked(pd64):
    with pytest.raises(TypeError, match="complex"):
        E.state_vel(torch.zeros(2, 64, 33), pd64, False)
    with pytest.raises(TypeError, match="complex"):
        E.lawson_rk4(torch.zeros(2, 64, 66, dtype=torch.float32), 0.1, 1, pd64)
    with pytest.raises(ValueError, match=r"n//2\+1"):
        E.state_vel(torch.zeros(2, 64, 64, dtype=torch.complex128), pd64, False)
    with pytest.raises(ValueError, match=r"n//2\+1"):
        E.integrate(torch.zeros(3, 64, 33, dtype=torch.complex128), 0.1, 1, pd64, "RK4")
    with pytest.raises(ValueError, match="snapshots"):
        turbulence.recurrence(torch.zeros(2, 64, 33, dtype=torch.complex128), pd64)


def test_forcing_of_another_grid_is_refused(pd64):
    with pytest.raises(ValueError, match="forcing"):
        C.get_context(pd64, 128, torch.float64)


def test_krylov_vectors_checked(built_lib):
    with pytest.raises(ValueError, match="inner"):
        linalg.gmres(lambda v: v, torch.ones(8, dtype=torch.float64), 129)
    with pytest.raises(ValueError, match="inner"):
        linalg.gmres(lambda v: v, torch.ones(8, dtype=torch.float64), 0)
    # host vectors never reach the cluster kernel
    with pytest.raises(ValueError, match="CUDA"):
        linalg.gmres(lambda v: v, torch.ones(8, dtype=torch.float64), 4)
    with pytest.raises(ValueError, match="CUDA"):
        linalg._vp(torch.ones(8, dtype=torch.float64))
    with pytest.raises(ValueError, match="outside a basis"):
        linalg._orth(torch.zeros(3, 8, dtype=torch.float64), 2, torch.ones(8), torch.zeros(5), 0)


def test_device_pointers_only():
    with pytest.raises(ValueError, match="GPU"):
        C.ptr(torch.zeros(4))
