"""ecs_linearize_jvp (primal solve overlapped with the tangent sweep) against
ecs_linearize followed by ecs_jvp.  Every kernel sees the same inputs in both
orders, so the objective, the tangents and the step statistics must be equal
bit for bit; the linearisation it leaves must serve later jvp calls."""
import numpy as np
import pytest
import torch

import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200.synthetic import initial_condition

pytestmark = pytest.mark.gpu

CASES = [
    # (mode, param kwargs, T): attempt caps that are multiples of 16 (the pipelined chunk) or not (sequential
    # fallback); fixed steps with a full record (pipelined) or checkpointed (sequential fallback)
    ("Lawson_RK43", dict(shift_reflect_ny=2, rot=False,
                         adaptive_dict={"atol": 1e-6, "checkpoints": 4, "max_steps_per_checkpoint": 32}), 0.3),
    ("Lawson_RK43", dict(shift_reflect_ny=5, rot=True,
                         adaptive_dict={"atol": 1e-9, "checkpoints": 2, "max_steps_per_checkpoint": 16}), 0.5),
    ("Lawson_RK43", dict(shift_reflect_ny=1, rot=False,
                         adaptive_dict={"atol": 1e-6, "checkpoints": 3, "max_steps_per_checkpoint": 7}), 0.2),
    ("Lawson_RK4", dict(num_checkpoints=2, ministeps=8, shift_reflect_ny=0, rot=False), 0.1),
    ("Lawson_RK4", dict(num_checkpoints=5, ministeps=15, shift_reflect_ny=3, rot=True), 0.4),   # 75 steps: 5 chunks
    ("Lawson_RK4", dict(num_checkpoints=4, ministeps=8, shift_reflect_ny=0, rot=False, ckpt_every=8), 0.2),
]


def _inputs(n, B):
    u0 = initial_condition(7, n, amp=6.0)
    rng = np.random.default_rng(5)
    du = np.stack([initial_condition(40 + i, n) * 0.1 + 0.01 * rng.standard_normal((2, n, n)) for i in range(B)])
    prim = {"fields": torch.as_tensor(u0, device="cuda"), "T": None, "sx": 0.21}
    tan = {"fields": torch.as_tensor(du, device="cuda"), "T": torch.linspace(-1.0, 1.0, B, dtype=torch.float64),
           "sx": torch.linspace(0.5, -0.5, B, dtype=torch.float64)}
    return prim, tan


@pytest.mark.parametrize("mode,kw,T", CASES)
def test_linearize_jvp_equals_sequential(cuda, mode, kw, T):
    n, B = 64, 8
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    prim, tan = _inputs(n, B)
    prim["T"] = T
    seq = E.Objective(pd, mode)
    seq.linearize(prim, force=True, batch=B)
    want_val = seq.last_value["fields"].clone()
    want_info = dict(seq.last_info)
    want = seq.jvp(prim, tan)
    want = {k: v.clone() for k, v in want.items()}

    pip = E.Objective(pd, mode)
    val, got = pip.linearize_jvp(prim, tan)
    torch.cuda.synchronize()
    assert pip.last_info == want_info
    assert torch.equal(val["fields"], want_val)
    for k in ("fields", "T", "sx"):
        assert torch.equal(got[k], want[k]), k
    # the linearisation left in the context serves a later jvp call
    again = pip.jvp(prim, tan)
    for k in ("fields", "T", "sx"):
        assert torch.equal(again[k], want[k]), k


@pytest.mark.parametrize("B", [34, 64])
def test_linearize_jvp_groups(cuda, B):
    """Batches of 32 or more tangents are swept as groups on several streams
    (three by default, one to four with ECS_TGROUPS); each tangent's result is the
    same as in the single sequential sweep."""
    n = 64
    kw = CASES[0][1]
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    prim, tan = _inputs(n, B)
    prim["T"] = 0.3
    seq = E.Objective(pd, "Lawson_RK43")
    seq.linearize(prim, force=True, batch=B)
    want = {k: v.clone() for k, v in seq.jvp(prim, tan).items()}
    got = E.Objective(pd, "Lawson_RK43").linearize_jvp(prim, tan)[1]
    for k in ("fields", "T", "sx"):
        assert torch.equal(got[k], want[k]), k


def test_linearize_jvp_repeated_calls(cuda):
    """Back-to-back pipelined calls on one context (graph and buffers reused)
    give the same result each time."""
    n, B = 64, 8
    kw = CASES[0][1]
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", **kw)
    prim, tan = _inputs(n, B)
    prim["T"] = 0.3
    obj = E.Objective(pd, "Lawson_RK43")
    first = obj.linearize_jvp(prim, tan)[1]["fields"].clone()
    for _ in range(2):
        assert torch.equal(obj.linearize_jvp(prim, tan)[1]["fields"], first)


@pytest.mark.parametrize("env", [{"ECS_ROWTAN_XT": "8"}, {"ECS_PDL_MINB": "8"}, {"ECS_TGROUPS": "1"},
                                 {"ECS_TGROUPS": "2"}])
def test_tuning_switches_do_not_change_results(cuda, env, monkeypatch):
    """The tuning switches (read when a context is created) change launch
    shapes and ordering only: the objective and a batch of 64 tangents at
    n = 128 are bit for bit those of the defaults."""
    from ecs_mhd_2d_b200 import context
    n, B = 128, 64
    kw = dict(shift_reflect_ny=0, rot=False, adaptive_dict={"atol": 1e-7, "checkpoints": 2, "max_steps_per_checkpoint": 32})
    pd = E.make_param_dict(n, 1 / 50, 1 / 50, forcing="kolmogorov+", **kw)
    prim, tan = _inputs(n, B)
    prim["T"] = 0.3

    def run():
        context.clear_cache()
        v, t = E.Objective(pd, "Lawson_RK43").linearize_jvp(prim, tan)
        return v["fields"].cpu().numpy(), t["fields"].cpu().numpy(), t["T"].cpu().numpy()

    base = run()
    for k, val in env.items():
        monkeypatch.setenv(k, val)
    other = run()
    monkeypatch.undo()
    context.clear_cache()
    for a, b in zip(base, other):
        assert np.array_equal(a, b)
