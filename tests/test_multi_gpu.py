"""Matvecs and gradients of several candidates in one sweep
(ecs_jvp_multi, ecs_loss_grad_multi).  Matvecs: every
candidate's objective and JVP equal those of its own single-candidate call
(Objective.linearize_jvp: the primal record then a tangent sweep), to 1e-13
relative (the two paths take the primal physical fields from different passes
of the same arithmetic), and match torch.func.jvp of the oracle to 1e-12.
Candidates differ in horizon, step count, T, sx, symmetry, state and tangent;
the longest runs past the others, which must stop at their own budget.
Gradients: every candidate's loss and gradient equal its own loss_and_grad
call and torch.func.vjp of the oracle's loss_RPO to 1e-12, with different
step counts (the reverse sweep is aligned at each candidate's end)."""
import numpy as np
import pytest
import torch
from torch.func import jvp as tjvp, vjp as tvjp

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200.synthetic import initial_condition
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_SAME = 1e-13
TOL_ORACLE = 1e-12

CANDS = [  # (num_checkpoints, ministeps, T, sx, shift_reflect_ny, rot)
    (2, 8, 0.08, 0.3, 0, False),
    (3, 8, 0.12, -0.2, 1, True),
    (1, 5, 0.03, 0.0, 2, False),
    (4, 8, 0.15, 0.7, 3, False),
    (2, 12, 0.1, -0.5, 0, True),
]


def _setup(n, dtype=torch.float64, re=40.0):
    rng = np.random.default_rng(4)
    prims, tans, pds, opds = [], [], [], []
    for i, (nc, ms, T, sx, ny, rot) in enumerate(CANDS):
        kw = dict(num_checkpoints=nc, ministeps=ms, shift_reflect_ny=ny, rot=rot)
        pds.append(E.make_param_dict(n, 1 / re, 1 / re, forcing="kolmogorov+", data_type=dtype, **kw))
        opds.append(O.make_param_dict(n, 1 / re, 1 / re, forcing="kolmogorov+", xp=O.TORCH, **kw))
        u = initial_condition(30 + i, n, amp=6.0)
        du = initial_condition(60 + i, n) * 0.1 + 0.01 * rng.standard_normal((2, n, n))
        prims.append({"fields": torch.as_tensor(u, dtype=dtype, device="cuda"), "T": T, "sx": sx})
        tans.append({"fields": torch.as_tensor(du, dtype=dtype, device="cuda"), "T": 0.3 - 0.2 * i, "sx": 0.1 * i - 0.2})
    return prims, tans, pds, opds


@pytest.mark.parametrize("n", [64, 128])
def test_jvp_multi_equals_single_candidate_calls(cuda, n):
    prims, tans, pds, _ = _setup(n)
    vals, jv = E.jvp_multi(prims, tans, pds)
    torch.cuda.synchronize()
    for b in range(len(CANDS)):
        v1, j1 = E.Objective(pds[b], "Lawson_RK4").linearize_jvp(prims[b], tans[b])
        assert rel_l2(vals[b]["fields"].cpu().numpy(), v1["fields"].cpu().numpy()) < TOL_SAME, b
        assert rel_l2(jv[b]["fields"].cpu().numpy(), j1["fields"].cpu().numpy()) < TOL_SAME, b
        for k in ("T", "sx"):
            w = float(j1[k])
            assert abs(float(jv[b][k]) - w) <= TOL_SAME * max(abs(w), 1e-30) + 1e-18, (k, b)


def test_jvp_multi_matches_oracle(cuda):
    n = 64
    prims, tans, pds, opds = _setup(n)
    vals, jv = E.jvp_multi(prims, tans, pds)
    for b in (1, 3):
        f = lambda d: O.objective_RPO(d, opds[b], "Lawson_RK4", xp=O.TORCH)
        p = {"fields": prims[b]["fields"].cpu(), "T": torch.tensor(prims[b]["T"], dtype=torch.float64),
             "sx": torch.tensor(prims[b]["sx"], dtype=torch.float64)}
        t = {"fields": tans[b]["fields"].cpu(), "T": torch.tensor(tans[b]["T"], dtype=torch.float64),
             "sx": torch.tensor(tans[b]["sx"], dtype=torch.float64)}
        wv, wt = tjvp(f, (p,), (t,))
        assert rel_l2(vals[b]["fields"].cpu().numpy(), wv["fields"].numpy()) < TOL_ORACLE, b
        assert rel_l2(jv[b]["fields"].cpu().numpy(), wt["fields"].numpy()) < TOL_ORACLE, b
        for k in ("T", "sx"):
            w = float(wt[k])
            assert abs(float(jv[b][k]) - w) <= TOL_ORACLE * max(abs(w), 1.0), (k, b)


def test_jvp_multi_repeated_and_reordered(cuda):
    """A second call reuses the captured step graph; candidates in another order
    (and a smaller batch) give each candidate the same result."""
    n = 64
    prims, tans, pds, _ = _setup(n)
    _, first = E.jvp_multi(prims, tans, pds)
    first = [j["fields"].clone() for j in first]
    order = [3, 0, 4]
    _, again = E.jvp_multi([prims[i] for i in order], [tans[i] for i in order], [pds[i] for i in order])
    for k, i in enumerate(order):
        assert rel_l2(again[k]["fields"].cpu().numpy(), first[i].cpu().numpy()) < TOL_SAME, i


def test_jvp_multi_fp32(cuda):
    """FP32 candidates against the FP64 oracle within FP32 rounding (5e-5)."""
    n = 64
    prims, tans, pds, opds = _setup(n, dtype=torch.float32)
    _, jv = E.jvp_multi(prims, tans, pds)
    b = 1
    f = lambda d: O.objective_RPO(d, opds[b], "Lawson_RK4", xp=O.TORCH)
    p = {"fields": prims[b]["fields"].double().cpu(), "T": torch.tensor(prims[b]["T"], dtype=torch.float64),
         "sx": torch.tensor(prims[b]["sx"], dtype=torch.float64)}
    t = {"fields": tans[b]["fields"].double().cpu(), "T": torch.tensor(tans[b]["T"], dtype=torch.float64),
         "sx": torch.tensor(tans[b]["sx"], dtype=torch.float64)}
    _, wt = tjvp(f, (p,), (t,))
    assert rel_l2(jv[b]["fields"].double().cpu().numpy(), wt["fields"].numpy()) < 5e-5


GCANDS = [  # (num_checkpoints, ministeps, T, sx, shift_reflect_ny, rot): step counts 16, 24, 32, 8 (segments of 8)
    (2, 8, 0.08, 0.3, 0, False),
    (3, 8, 0.12, -0.2, 1, True),
    (4, 8, 0.15, 0.7, 3, False),
    (1, 8, 0.03, 0.0, 2, False),
]


def _gsetup(n, cands, re=40.0):
    xs, pds, opds = [], [], []
    for i, (nc, ms, T, sx, ny, rot) in enumerate(cands):
        kw = dict(num_checkpoints=nc, ministeps=ms, shift_reflect_ny=ny, rot=rot)
        pds.append(E.make_param_dict(n, 1 / re, 1 / re, forcing="kolmogorov+", **kw))
        opds.append(O.make_param_dict(n, 1 / re, 1 / re, forcing="kolmogorov+", xp=O.TORCH, **kw))
        xs.append({"fields": torch.as_tensor(initial_condition(40 + i, n, amp=6.0), device="cuda"), "T": T, "sx": sx})
    return xs, pds, opds


@pytest.mark.parametrize("n,cands", [(64, GCANDS), (128, GCANDS[:3]), (64, CANDS)])
def test_loss_grad_multi_equals_single_candidate_calls(cuda, n, cands):
    """Each candidate's loss and gradient equal its own loss_and_grad call
    (the single-candidate adjoint) to 1e-12; the third case has step counts
    16, 24, 5, 32, 24 (segments of one step)."""
    xs, pds, _ = _gsetup(n, cands)
    res = E.loss_grad_multi(xs, pds)
    for b in range(len(cands)):
        (l1, _), g1 = E.loss_and_grad(xs[b], pds[b], "Lawson_RK4")
        lb, gb = res[b]
        assert abs(float(lb) - float(l1)) <= 1e-12 * abs(float(l1)), b
        assert rel_l2(gb["fields"].cpu().numpy(), g1["fields"].cpu().numpy()) < 1e-12, b
        for k in ("T", "sx"):
            w = float(g1[k])
            assert abs(float(gb[k]) - w) <= 1e-12 * max(abs(w), 1.0), (k, b)


def test_loss_grad_multi_matches_oracle(cuda):
    """Against torch.func.vjp of the oracle's loss_RPO (as jax.value_and_grad): 1e-12."""
    n = 64
    xs, pds, opds = _gsetup(n, GCANDS)
    res = E.loss_grad_multi(xs, pds)
    for b in (1, 2):
        f = lambda d: O.loss_RPO(d, opds[b], "Lawson_RK4", xp=O.TORCH)[0]
        p = {"fields": xs[b]["fields"].cpu(), "T": torch.tensor(xs[b]["T"], dtype=torch.float64),
             "sx": torch.tensor(xs[b]["sx"], dtype=torch.float64)}
        lw, fn = tvjp(f, p)
        gw = fn(torch.tensor(1.0, dtype=torch.float64))[0]
        lb, gb = res[b]
        assert abs(float(lb) - float(lw)) <= 1e-12 * abs(float(lw))
        assert rel_l2(gb["fields"].cpu().numpy(), gw["fields"].numpy()) < 1e-12, b
        for k in ("T", "sx"):
            w = float(gw[k])
            assert abs(float(gb[k]) - w) <= 1e-12 * max(abs(w), 1.0), (k, b)
