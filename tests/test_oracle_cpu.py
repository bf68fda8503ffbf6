"""The oracle against the reference's golden data and self-check properties (CPU only)."""
import json
import os

import numpy as np
import pytest
import torch

import oracle as O
from conftest import GOLDEN, rel_l2
from ecs_mhd_2d_b200.synthetic import initial_condition


def solution_pd(d, xp=O.NUMPY):
    n = d["fields"].shape[-1]
    return O.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=d["b0"], xp=xp,
                             num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
                             shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))


@pytest.mark.parametrize("name", ["Re40_RPO6", "Re40_TW1"])
def test_reference_solutions_close_under_oracle(name):
    """Converged reference solutions satisfy |g.Phi_T(u0) - u0| / |u0| << 1 (reference README step 3)."""
    d = np.load(os.path.join(GOLDEN, f"solution_{name}.npz"))
    out = O.objective_RPO({"fields": d["fields"], "T": float(d["T"]), "sx": float(d["sx"])}, solution_pd(d),
                          "Lawson_RK4")
    r = np.linalg.norm(out["fields"]) / np.linalg.norm(d["fields"])
    assert r < 1e-8
    assert abs(r - float(d["closure"])) <= 1e-12 + 1e-6 * float(d["closure"])


def test_closure_record_covers_all_reference_solutions():
    rec = json.load(open(os.path.join(GOLDEN, "closure_lawson_rk4.json")))
    assert len(rec) == 15
    assert max(v["closure"] for v in rec.values()) < 1e-7


def test_synthetic_golden_reproduces():
    g = np.load(os.path.join(GOLDEN, "synthetic_n64.npz"))
    n = 64
    assert np.array_equal(initial_condition(int(g["seed"]), n), g["u0"])
    pd = O.make_param_dict(n, float(g["nu"]), float(g["eta"]), forcing="kolmogorov+",
                           num_checkpoints=2, ministeps=32, shift_reflect_ny=1, rot=True)
    f0 = np.fft.rfft2(g["u0"])
    assert rel_l2(O.state_vel(f0, pd, False), g["state_vel"]) < 1e-14
    out = O.objective_RPO({"fields": g["u0"], "T": 0.32, "sx": 0.3}, pd, "Lawson_RK4")
    assert rel_l2(out["fields"], g["objective"]) < 1e-13


def test_numpy_and_torch_restatements_agree():
    n = 64
    u0 = initial_condition(4, n)
    kw = dict(num_checkpoints=1, ministeps=8, shift_reflect_ny=3, rot=True)
    pn = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    pt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **kw)
    a = O.objective_RPO({"fields": u0, "T": 0.1, "sx": 0.2}, pn, "Lawson_RK4")["fields"]
    b = O.objective_RPO({"fields": torch.from_numpy(u0), "T": torch.tensor(0.1, dtype=torch.float64),
                         "sx": torch.tensor(0.2, dtype=torch.float64)}, pt, "Lawson_RK4", xp=O.TORCH)["fields"]
    assert rel_l2(b.numpy(), a) < 1e-13


def test_lawson_rk4_fourth_order():
    """Temporal order ~4 (the reference's RK4 order check, mhd_jax.py:278-292)."""
    n = 64
    pd = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+")
    f0 = np.fft.rfft2(initial_condition(0, n))
    v = lambda f: O.state_vel(f, pd, False)
    L = O.dissipation(pd)
    t = 0.2
    fine = O.lawson_rk4(f0, t, 512, v, L, pd["mask"])
    steps = np.array([32, 64, 128])
    err = [np.linalg.norm(np.fft.irfft2(O.lawson_rk4(f0, t, int(s), v, L, pd["mask"]) - fine)) for s in steps]
    slope = np.polyfit(np.log(steps), np.log(err), 1)[0]
    assert -4.6 < slope < -3.4


@pytest.mark.parametrize("ny,rot", [(0, True), (1, False), (5, True)])
def test_symmetry_equivariance(ny, rot):
    """g.Phi_T = Phi_T.g for the shift-reflect/rotation subgroup (symmetry.py:58-127)."""
    n = 64
    pd = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov")
    f0 = np.fft.rfft2(initial_condition(1, n))
    v = lambda f: O.state_vel(f, pd, False)
    L = O.dissipation(pd)
    g = lambda f: (O.rot180(O.shift_reflect(f, ny, pd)) if rot else O.shift_reflect(f, ny, pd))
    a = g(O.lawson_rk4(f0, 0.05, 10, v, L, pd["mask"]))
    b = O.lawson_rk4(g(f0), 0.05, 10, v, L, pd["mask"])
    assert rel_l2(np.fft.irfft2(a), np.fft.irfft2(b)) < 1e-12


def test_lawson_rk6_sixth_order():
    """Lawson_RK6 (timestepping.py:83-125) converges at order ~6."""
    n = 64
    pd = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+")
    f0 = np.fft.rfft2(initial_condition(0, n, amp=3.0))
    v = lambda f: O.state_vel(f, pd, False)
    L = O.dissipation(pd)
    t = 0.2
    fine = O.lawson_rk6(f0, t, 256, v, L, pd["mask"])
    steps = np.array([16, 24, 32])
    err = [np.linalg.norm(np.fft.irfft2(O.lawson_rk6(f0, t, int(s), v, L, pd["mask"]) - fine)) for s in steps]
    slope = np.polyfit(np.log(steps), np.log(err), 1)[0]
    assert -7.0 < slope < -5.0, err


def test_state_vel_jvp_matches_autodiff():
    """The written-out forward derivative of state_vel equals torch.func.jvp of
    its torch restatement (the two stand-ins for jax.jvp in tdrk4)."""
    n = 64
    pn = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+")
    pt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH)
    f = np.fft.rfft2(initial_condition(2, n))
    k = np.fft.rfft2(initial_condition(3, n, amp=1.0))
    for diss in (False, True):
        a = O.state_vel_jvp(f, k, pn, diss)
        b = torch.func.jvp(lambda x: O.state_vel(x, pt, diss, O.TORCH), (torch.from_numpy(f),),
                           (torch.from_numpy(k),))[1].numpy()
        assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b)


def test_tdrk4_fourth_order_and_backends_agree():
    """TDRK4 (timestepping.py:127-149) converges at order ~4; the numpy and torch
    restatements agree."""
    n = 64
    kw = dict(num_checkpoints=1, ministeps=16, shift_reflect_ny=0, rot=False)
    pd = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    f0 = np.fft.rfft2(initial_condition(0, n))
    v = lambda f: O.state_vel(f, pd, True)
    jac = lambda f, k: O.state_vel_jvp(f, k, pd, True)
    t = 0.1
    fine = O.tdrk4(f0, t, 512, v, jac)
    steps = np.array([32, 64, 128])
    err = [np.linalg.norm(np.fft.irfft2(O.tdrk4(f0, t, int(s), v, jac) - fine)) for s in steps]
    slope = np.polyfit(np.log(steps), np.log(err), 1)[0]
    assert -4.7 < slope < -3.3, err
    pt = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", xp=O.TORCH, **kw)
    u0 = initial_condition(4, n)
    a = O.objective_RPO({"fields": u0, "T": 0.1, "sx": 0.2}, pd, "TDRK4")["fields"]
    b = O.objective_RPO({"fields": torch.from_numpy(u0), "T": torch.tensor(0.1, dtype=torch.float64),
                         "sx": torch.tensor(0.2, dtype=torch.float64)}, pt, "TDRK4", xp=O.TORCH)["fields"]
    assert rel_l2(b.detach().numpy(), a) < 1e-13
