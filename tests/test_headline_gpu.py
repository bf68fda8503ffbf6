"""Oracle parity of the exact code paths that the benchmark lines time, at their
own grid sizes.

* Config 1 (the headline matvec batch): ``Objective.linearize_jvp`` at n=128
  FP64, Re=Rm=50, Lawson_RK43 atol 1e-8 with a 64 x 64 attempt cap, a batch of
  64 unit-norm tangents (three tangent stream groups, the 4-row tangent row
  tiles of n=128).  Tangents from every group are compared with
  ``torch.func.jvp`` of the oracle (as jax.jvp of objective_RPO,
  jax_scripts/lib/utils.py:108), and the accept/reject sequence with the
  oracle's.  Horizon T=0.5 keeps the oracle cheap and still contains rejected
  attempts (145 accepted, 6 rejected); the full horizon T=4.6 is checked
  through the objective value, the step counts, one tangent, and
  JVP/VJP adjointness.
* Config 2 (the adjoint gradient): ``loss_and_grad(normalized=True)`` and
  ``ecs_vjp`` at n=128, Re=40, Lawson_RK4 with dt = 4.26/1088 and checkpoints
  every 32 steps (jax.checkpoint per segment, loss_functions.py:63), 96 steps
  = 3 recomputed segments, against ``torch.func.vjp`` of the oracle.
* Config 0 (plain forward integration): n=64, Re=40, 1024 Lawson-RK4 steps of
  dt=0.005 for the bench's 8 seeded states, against the numpy oracle.

Tolerances (relative L2, written beside each check):
* Lawson-RK4 paths: 1e-12.  After 1024 steps the
  oracle's numpy and torch forms differ by <= 1.2e-14, so 1e-12 leaves two
  orders of magnitude for the kernels' different summation order.
* Lawson-RK4(3) paths: 1e-10.  The controller's error estimate is a difference
  of nearly equal stage derivatives; a 1e-12 relative change in it moves the
  objective by ~6e-12, and the oracle's own numpy and torch forms differ by
  6-8e-12.  The accept/reject sequence must be identical.
"""
import os

import numpy as np
import pytest
import torch
from torch.func import jvp as tjvp, vjp as tvjp

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200.synthetic import initial_condition, unit_tangents
from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu

TOL_RK4 = 1e-12
TOL_43 = 1e-10

# config 1 (bench.py's workload)
N1, RE1, SX1, ATOL1, CAP1, B1 = 128, 50.0, 0.12, 1e-8, (64, 64), 64
# config 2
N2, RE2, DT2 = 128, 40.0, 4.26 / 1088


@pytest.fixture(scope="module", autouse=True)
def _threads():
    torch.set_num_threads(max(1, os.cpu_count() or 1))


def _cfg1_kw():
    return dict(shift_reflect_ny=0, rot=False,
                adaptive_dict={"atol": ATOL1, "checkpoints": CAP1[0], "max_steps_per_checkpoint": CAP1[1]})


def _cfg1_inputs():
    u0 = initial_condition(0, N1, amp=2.0)
    tv = unit_tangents(0, N1, B1)
    return u0, tv


def _oracle_jvp(pdt, mode, u0, T, sx, t):
    f = lambda d: O.objective_RPO(d, pdt, mode, xp=O.TORCH)
    prim = {"fields": torch.from_numpy(u0), "T": torch.tensor(T, dtype=torch.float64),
            "sx": torch.tensor(sx, dtype=torch.float64)}
    tan = {"fields": torch.from_numpy(np.ascontiguousarray(t[1:-1].reshape(2, *u0.shape[1:]))),
           "T": torch.tensor(t[0], dtype=torch.float64), "sx": torch.tensor(t[-1], dtype=torch.float64)}
    val, out = tjvp(f, (prim,), (tan,))
    return {k: v.detach().numpy() for k, v in val.items()}, {k: v.detach().numpy() for k, v in out.items()}


def _headline(T):
    u0, tv = _cfg1_inputs()
    pd = E.make_param_dict(N1, 1 / RE1, 1 / RE1, forcing="kolmogorov+", **_cfg1_kw())
    obj = E.Objective(pd, "Lawson_RK43")
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": SX1}
    tan = {"fields": torch.as_tensor(tv[:, 1:-1].reshape(B1, 2, N1, N1), device="cuda").contiguous(),
           "T": torch.as_tensor(tv[:, 0]), "sx": torch.as_tensor(tv[:, -1])}
    val, out = obj.linearize_jvp(prim, tan)
    torch.cuda.synchronize()
    return u0, tv, pd, obj, prim, tan, val, out


def _check_steps(obj, u0, T):
    opd = O.make_param_dict(N1, 1 / RE1, 1 / RE1, forcing="kolmogorov+", **_cfg1_kw())
    _, _, info = O.mismatch_RPO({"fields": u0, "T": T, "sx": SX1}, opd, "Lawson_RK43")
    assert obj.last_info["completed"] and info["completed"]
    assert (obj.last_info["accepted"], obj.last_info["rejected"]) == (info["accepted"], info["rejected"])
    return opd, info


def test_headline_jvp_batch_matches_oracle(cuda):
    """Tangents 0, 21, 42 and 63 of the bench's 64-tangent sweep (one in each of
    the three stream groups, plus the last) against torch.func.jvp of the oracle
    at T=0.5: 1e-10 on the fields, the phase-condition rows and the objective."""
    T = 0.5
    u0, tv, pd, obj, prim, tan, val, out = _headline(T)
    opd, info = _check_steps(obj, u0, T)
    assert info["rejected"] > 0          # the rejected-attempt path is part of the check
    pdt = O.make_param_dict(N1, 1 / RE1, 1 / RE1, forcing="kolmogorov+", xp=O.TORCH, **_cfg1_kw())
    for b in (0, 21, 42, 63):
        assert abs(tv[b, 0]) > 0 and abs(tv[b, -1]) > 0
        wv, wt = _oracle_jvp(pdt, "Lawson_RK43", u0, T, SX1, tv[b])
        if b == 0:
            assert rel_l2(val["fields"].cpu().numpy(), wv["fields"]) < TOL_43
        assert rel_l2(out["fields"][b].cpu().numpy(), wt["fields"]) < TOL_43, b
        for k in ("T", "sx"):
            w = float(wt[k])
            assert abs(float(out[k][b]) - w) <= TOL_43 * max(abs(w), 1e-30), (k, b)


def test_headline_full_horizon(cuda):
    """The bench workload itself (T=4.6, 1983 accepted + 5 rejected attempts):
    objective value and step counts against the numpy oracle (1e-10, identical
    counts); tangent 0 of the batch against the committed torch.func.jvp of the
    oracle at this workload (tests/golden/headline_jvp_n128.npz, made by
    make_golden.py headline: minutes of CPU time; 1e-10); and
    <u, J v_b> = <J^T u, v_b> for two batch tangents (1e-11)."""
    T = 4.6
    u0, tv, pd, obj, prim, tan, val, out = _headline(T)
    opd, info = _check_steps(obj, u0, T)
    want = O.objective_RPO({"fields": u0, "T": T, "sx": SX1}, opd, "Lawson_RK43")
    assert rel_l2(val["fields"].cpu().numpy(), want["fields"]) < TOL_43
    gold = np.load(os.path.join(GOLDEN, "headline_jvp_n128.npz"))
    assert (int(gold["accepted"]), int(gold["rejected"])) == (info["accepted"], info["rejected"])
    assert rel_l2(want["fields"], gold["objective"]) < TOL_43          # the fixture is of this oracle
    assert rel_l2(out["fields"][0].cpu().numpy(), gold["jvp_fields"]) < TOL_43
    for k in ("T", "sx"):
        w = float(gold["jvp_" + k])
        assert abs(float(out[k][0]) - w) <= TOL_43 * max(abs(w), 1e-30), k
    rng = np.random.default_rng(17)
    u = {"fields": torch.as_tensor(rng.standard_normal((2, N1, N1)), device="cuda"), "T": 0.4, "sx": -0.9}
    _, jacT = E.vjp(obj, prim)
    g = jacT(u)[0]
    for b in (5, 50):
        lhs = float(torch.sum(u["fields"] * out["fields"][b])) + 0.4 * float(out["T"][b]) - 0.9 * float(out["sx"][b])
        rhs = (float(torch.sum(g["fields"] * tan["fields"][b])) + float(tan["T"][b]) * float(g["T"])
               + float(tan["sx"][b]) * float(g["sx"]))
        assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), abs(rhs)), b


def test_headline_batch_equals_single_tangent(cuda):
    """A tangent pushed through the 64-wide, three-group sweep equals the same
    tangent pushed alone at the same linearisation (1e-14: the two runs use
    different row tiles and groupings of the same per-element arithmetic)."""
    T = 0.5
    u0, tv, pd, obj, prim, tan, val, out = _headline(T)
    for b in (0, 40):
        one = obj.jvp(prim, {"fields": tan["fields"][b].contiguous(), "T": float(tan["T"][b]),
                             "sx": float(tan["sx"][b])})
        assert rel_l2(one["fields"].cpu().numpy(), out["fields"][b].cpu().numpy()) < 1e-14, b


def _cfg2(steps):
    nc = steps // 32
    kw = dict(num_checkpoints=nc, ministeps=32, shift_reflect_ny=0, rot=False)
    pd = E.make_param_dict(N2, 1 / RE2, 1 / RE2, forcing="kolmogorov+", ckpt_every=32, **kw)
    pdt = O.make_param_dict(N2, 1 / RE2, 1 / RE2, forcing="kolmogorov+", xp=O.TORCH, **kw)
    return pd, pdt, steps * DT2


def test_config2_gradient_matches_oracle(cuda):
    """The bench's config-2 gradient (normalised loss |shift(u(T)) - u(0)|^2 / |u(0)|^2,
    checkpoints every 32 steps, recomputation in between) over 3 segments (96 steps
    of dt = 4.26/1088) against torch.func.vjp of the oracle: 1e-12."""
    pd, pdt, T = _cfg2(96)
    u0 = initial_condition(2, N2, amp=2.0)
    sx = 0.1
    (loss, _), g = E.loss_and_grad({"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": sx}, pd,
                                   "Lawson_RK4", normalized=True)

    def lossn(d):
        l, _ = O.loss_RPO(d, pdt, "Lawson_RK4", xp=O.TORCH)
        return l * (2 * N2 * N2) / torch.sum(d["fields"] ** 2)

    prim = {"fields": torch.from_numpy(u0), "T": torch.tensor(T, dtype=torch.float64),
            "sx": torch.tensor(sx, dtype=torch.float64)}
    lw, fn = tvjp(lossn, prim)
    gw = fn(torch.tensor(1.0, dtype=torch.float64))[0]
    assert abs(float(loss) - float(lw)) <= TOL_RK4 * abs(float(lw))
    assert rel_l2(g["fields"].cpu().numpy(), gw["fields"].numpy()) < TOL_RK4
    for k in ("T", "sx"):
        w = float(gw[k])
        assert abs(float(g[k]) - w) <= TOL_RK4 * max(abs(w), 1e-30), k


def test_config2_vjp_matches_oracle(cuda):
    """ecs_vjp of objective_RPO at the config-2 settings (checkpoints every 32, 96
    steps) for two cotangents against torch.func.vjp of the oracle: 1e-12."""
    pd, pdt, T = _cfg2(96)
    u0 = initial_condition(2, N2, amp=2.0)
    sx = 0.1
    rng = np.random.default_rng(23)
    cf = rng.standard_normal((2, 2, N2, N2))
    cT, csx = np.array([0.6, -1.1]), np.array([0.3, 0.0])
    obj = E.Objective(pd, "Lawson_RK4")
    _, jacT = E.vjp(obj, {"fields": torch.as_tensor(u0, device="cuda"), "T": T, "sx": sx})
    got = jacT({"fields": torch.as_tensor(cf, device="cuda"), "T": torch.as_tensor(cT),
                "sx": torch.as_tensor(csx)})[0]
    f = lambda d: O.objective_RPO(d, pdt, "Lawson_RK4", xp=O.TORCH)
    prim = {"fields": torch.from_numpy(u0), "T": torch.tensor(T, dtype=torch.float64),
            "sx": torch.tensor(sx, dtype=torch.float64)}
    _, fn = tvjp(f, prim)
    for b in range(2):
        w = fn({"fields": torch.from_numpy(cf[b]), "T": torch.tensor(cT[b], dtype=torch.float64),
                "sx": torch.tensor(csx[b], dtype=torch.float64)})[0]
        assert rel_l2(got["fields"][b].cpu().numpy(), w["fields"].numpy()) < TOL_RK4, b
        for k in ("T", "sx"):
            assert abs(float(got[k][b]) - float(w[k])) <= TOL_RK4 * max(abs(float(w[k])), 1.0), (k, b)


def test_config0_1024_steps_match_oracle(cuda):
    """The bench's config-0 run (8 seeded states, n=64, Re=40, 1024 Lawson-RK4
    steps of dt=0.005, one batched call) against the numpy oracle per state: 1e-12."""
    n, S, dt = 64, 1024, 0.005
    u = np.stack([initial_condition(s, n) for s in range(8)])
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+")
    opd = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+")
    f0 = torch.as_tensor(np.fft.rfft2(u), device="cuda")
    got = E.lawson_rk4(f0, S * dt, S, pd).cpu().numpy()
    v = lambda x: O.state_vel(x, opd, False)
    L = O.dissipation(opd)
    for s in range(8):
        want = O.lawson_rk4(np.fft.rfft2(u[s]), S * dt, S, v, L, opd["mask"])
        assert rel_l2(np.fft.irfft2(got[s], s=(n, n)), np.fft.irfft2(want, s=(n, n))) < TOL_RK4, s
