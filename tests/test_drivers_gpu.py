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
from ecs_mhd_2d_b200.utils import relative_error_RPO

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


def test_mixed_precision_newton_tracks_fp64(cuda):
    """Newton-GMRES with FP32 Jacobian products (FP64 residuals, Arnoldi and
    least squares) follows the all-FP64 iteration: the same residual after
    each step to within 2 %, and the residual falls every step."""
    x, pd = perturbed_rpo6(1e-4)
    _, h32 = drivers.mixed_precision_newton(x, pd, "Lawson_RK4", iters=2, inner=16, refine=0)
    x, pd = perturbed_rpo6(1e-4)
    h64 = []
    for _ in range(2):
        x, st = drivers.newton_gmres_update(x, pd, "Lawson_RK4", inner=16, use_transpose=True)
        h64.append(st)
    x = drivers._as_device_dict(x)
    e64 = float(relative_error_RPO(x, E.objective_RPO(x, pd, "Lawson_RK4")))
    r32 = [h["rel_err"] for h in h32[:-1]] + [h32[-1]["final_rel_err"]]
    assert all(b < a for a, b in zip(r32, r32[1:])), h32
    for a, b in zip(r32[:2], [h["rel_err"] for h in h64]):
        assert abs(a - b) <= 0.02 * b, (h32, h64)
    assert abs(r32[-1] - e64) <= 0.02 * e64, (r32, e64)


def test_mixed_precision_newton_reaches_1e10_at_n256(cuda):
    """The mixed-precision target at 256^2 (Re=50): the reference's RPO2
    (solutions/Re50/RPO2.npz, 768 Lawson-RK4 steps) perturbed by 1e-7, four
    Newton-GMRES steps with FP32 stepping and FP32 JVP/VJP products (FP64
    residuals, Arnoldi and Hessenberg least squares), then two FP64 refinement
    steps (jax_scripts/newton.py:151-215); 32 Krylov vectors on the normal
    equations cut the residual about 7x per step here.  The final relative residual
    |objective| / |fields| is <= 1e-10 as evaluated by the FP64 numpy oracle,
    and the device's FP64 residual agrees with the oracle's to 1e-12
    (absolute, on a relative residual)."""
    import oracle as O
    d = np.load("tests/golden/solution_Re50_RPO2.npz")
    n = d["fields"].shape[-1]
    kw = dict(num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
              shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))
    pd = E.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=d["b0"], forcing="kolmogorov", **kw)
    u = E.dealias(torch.as_tensor(d["fields"] + 1e-7 * initial_condition(98, n, amp=1.0), device="cuda"), pd)
    x0 = {"fields": u, "T": float(d["T"]) * (1 + 1e-7), "sx": float(d["sx"])}
    r0 = float(relative_error_RPO(x0, E.objective_RPO(x0, pd, "Lawson_RK4")))
    x, hist = drivers.mixed_precision_newton(x0, pd, "Lawson_RK4", iters=4, inner=32, refine=2)
    assert [h["jacobian"] for h in hist[:-1]] == ["fp32"] * 4 + ["fp64"] * 2
    r_dev = hist[-1]["final_rel_err"]
    opd = O.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=tuple(d["b0"]), forcing="kolmogorov", **kw)
    xh = {"fields": x["fields"].cpu().numpy(), "T": float(x["T"]), "sx": float(x["sx"])}
    fo = O.objective_RPO(xh, opd, "Lawson_RK4")["fields"]
    r_orc = float(np.linalg.norm(fo) / np.linalg.norm(xh["fields"]))
    assert r0 > 1e-8 and r_orc <= 1e-10, (r0, r_orc, hist)
    assert abs(r_dev - r_orc) <= 1e-12, (r_dev, r_orc)


def test_newton_gmres_tdrk4_reference_default(cuda):
    """The reference Newton driver's default configuration (mode "TDRK4",
    use_transpose=True; jax_scripts/newton.py:70, :151-215) on the reference's
    TW1 -- converged with TDRK4 -- perturbed off the orbit: one step shrinks
    the residual sharply."""
    d = np.load("tests/golden/solution_Re40_TW1.npz")
    n = d["fields"].shape[-1]
    pd = E.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=d["b0"], forcing="kolmogorov",
                           num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
                           shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))
    u = torch.as_tensor(d["fields"] + 1e-4 * initial_condition(98, n, amp=1.0), device="cuda")
    x = {"fields": E.dealias(u, pd), "T": float(d["T"]) * (1 + 1e-4), "sx": float(d["sx"])}
    f0 = float(torch.linalg.norm(E.objective_RPO(x, pd, "TDRK4")["fields"]))
    new, st = drivers.newton_gmres_update(x, pd, "TDRK4", inner=16, use_transpose=True)
    f1 = float(torch.linalg.norm(E.objective_RPO(new, pd, "TDRK4")["fields"]))
    assert f1 < 0.1 * f0, (f0, f1, st)


def test_floquet_neutral_directions_and_power_iteration(cuda):
    """For the reference's TW1 (converged with TDRK4) the Floquet map of
    jax_scripts/floquet.py has multiplier 1 along the flow and along the
    x-shift (symmetry directions), to the orbit's closure accuracy; a short
    block power iteration gives a finite Schur factor with those multipliers
    among its eigenvalues' neighbourhood of 1."""
    d = np.load("tests/golden/solution_Re40_TW1.npz")
    n = d["fields"].shape[-1]
    pd = E.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=d["b0"], forcing="kolmogorov",
                           num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
                           shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))
    x = {"fields": torch.as_tensor(d["fields"], device="cuda"), "T": float(d["T"]), "sx": float(d["sx"])}
    apply = drivers.floquet_operator(x, pd, "TDRK4")
    f0 = torch.fft.rfft2(x["fields"])
    kx = torch.fft.fftfreq(n, 1 / n, dtype=torch.float64, device="cuda").reshape(-1, 1)
    vx = torch.fft.irfft2(1j * kx * f0, s=(n, n))                        # d/dx u0 (shift direction)
    vt = E.state_vel(f0, pd, include_dissipation=True)                   # d/dt u0 (flow direction)
    vt = torch.fft.irfft2(vt, s=(n, n))
    for v in (vx, vt):
        v = E.dealias(v.contiguous(), pd)
        jv = apply(v.unsqueeze(0))[0]
        assert float(torch.linalg.norm(jv - v) / torch.linalg.norm(v)) < 1e-6
    R, Q = drivers.floquet_power_iteration(x, pd, "TDRK4", block_size=4, maxit=3, seed=0)
    assert R.shape == (4, 4) and bool(torch.isfinite(R).all())
    G = Q.reshape(4, -1) @ Q.reshape(4, -1).T
    assert float(torch.linalg.norm(G - torch.eye(4, dtype=G.dtype, device=G.device))) < 1e-12
