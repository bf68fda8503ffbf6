"""The cluster-resident tangent sweep (k_tan_chain: one launch runs the pass
list of the adaptive Lawson-RK4(3) JVP -- column stages, row passes, updates of
rejected attempts) against the launch-per-pass sweep (ECS_CHAIN_MAXB=0).  Both
run the same per-column and per-row bodies in the same order, so the JVP of
objective_RPO (jax.jvp at jax_scripts/lib/utils.py:108) is equal bit for bit:
with rejected attempts, with regeneration-chunk boundaries inside the list
(ECS_REGEN_ITEMS), for one and for several tangents, at n = 64 and 128, with
the passes exchanging their intermediate arrays through distributed shared
memory and through global memory (ECS_CHAIN_DSMEM), with 8- and 16-warp CTAs
(ECS_CHAIN_WARPS), and with the tangent slots in shared or global memory
(ECS_CHAIN_DSLOTS)."""
import numpy as np
import pytest
import torch

import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import context
from ecs_mhd_2d_b200.synthetic import initial_condition

pytestmark = pytest.mark.gpu

CASES = [   # (n, B, T, atol, amp, env)
    (64, 1, 0.3, 1e-6, 6.0, {}),
    (64, 3, 0.3, 1e-6, 6.0, {"ECS_REGEN_ITEMS": "8"}),
    (64, 64, 0.2, 1e-7, 6.0, {"ECS_REGEN_ITEMS": "24"}),
    (128, 1, 0.15, 1e-8, 2.0, {}),
    (128, 5, 0.15, 1e-8, 2.0, {"ECS_REGEN_ITEMS": "16"}),
    # the 128^2 matvec workload's trajectory (initial condition seed 0, 64 x 64
    # attempt cap) over T = 0.5: 145 accepted and 6 rejected attempts
    (128, 2, 0.5, 1e-8, 2.0, {"ECS_REGEN_ITEMS": "64", "seed": 0}),
]


# (warps per CTA, exchange through distributed shared memory, tangent slots in shared memory)
VARIANTS = [(8, 1, 1), (8, 0, 1), (8, 1, 0), (8, 0, 0), (16, 1, 0), (16, 0, 0)]


def _run(n, B, T, atol, amp, env, monkeypatch, chain, variant=(8, 1, 1)):
    env = dict(env, ECS_CHAIN_WARPS=str(variant[0]), ECS_CHAIN_DSMEM=str(variant[1]), ECS_CHAIN_DSLOTS=str(variant[2]))
    seed = env.pop("seed", 4)
    cap = (64, 64) if seed == 0 else (4, 64)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    if chain:
        monkeypatch.setenv("ECS_CHAIN_MINB", "1")
        monkeypatch.setenv("ECS_CHAIN_MAXB", "64")
    else:
        monkeypatch.setenv("ECS_CHAIN_MAXB", "0")
    context.clear_cache()
    try:
        pd = E.make_param_dict(n, 1 / 50, 1 / 50, forcing="kolmogorov+", shift_reflect_ny=1, rot=False,
                               adaptive_dict={"atol": atol, "checkpoints": cap[0], "max_steps_per_checkpoint": cap[1]})
        rng = np.random.default_rng(3)
        prim = {"fields": torch.as_tensor(initial_condition(seed, n, amp=amp), device="cuda"), "T": T, "sx": 0.2}
        du = np.stack([initial_condition(60 + i, n) * 0.1 + 0.01 * rng.standard_normal((2, n, n)) for i in range(B)])
        tan = {"fields": torch.as_tensor(du, device="cuda"), "T": torch.linspace(-0.7, 1.1, B, dtype=torch.float64),
               "sx": torch.linspace(0.4, -0.3, B, dtype=torch.float64)}
        obj = E.Objective(pd, "Lawson_RK43")
        obj.linearize(prim, force=True, batch=B)
        ctx = context.get_context(pd, n, torch.float64, B)
        torch.cuda.synchronize()
        c0 = ctx.lib.ecs_launch_count(ctx.handle)
        out = obj.jvp(prim, tan)
        torch.cuda.synchronize()
        launches = ctx.lib.ecs_launch_count(ctx.handle) - c0
        res = {k: v.detach().cpu().clone() for k, v in out.items()}
        return res, dict(obj.last_info), launches
    finally:
        monkeypatch.undo()
        context.clear_cache()


@pytest.mark.parametrize("n,B,T,atol,amp,env", CASES)
def test_chain_equals_launch_per_pass(cuda, monkeypatch, n, B, T, atol, amp, env):
    want, info, per_pass = _run(n, B, T, atol, amp, env, monkeypatch, chain=False)
    for v in VARIANTS:
        got, info2, chained = _run(n, B, T, atol, amp, env, monkeypatch, chain=True, variant=v)
        assert info == info2
        for k in ("fields", "T", "sx"):
            assert torch.equal(got[k], want[k]), (k, v)
        # the pass list ran as a handful of launches instead of one per pass
        assert chained < per_pass // 4, (chained, per_pass)


def test_chain_covers_rejected_attempts(cuda, monkeypatch):
    """The last case's trajectory rejects attempts, so the list's reject
    updates are part of the comparison."""
    _, info, _ = _run(*CASES[-1], monkeypatch, chain=True)
    assert info["rejected"] > 0, info


RK4_CASES = [(64, 1, 5), (64, 8, 40), (128, 1, 37), (128, 3, 16)]   # (n, B, steps)


def _rk4(n, B, steps, monkeypatch, chain, variant=(8, 1, 1)):
    monkeypatch.setenv("ECS_CHAIN_WARPS", str(variant[0]))
    monkeypatch.setenv("ECS_CHAIN_DSMEM", str(variant[1]))
    if chain:
        monkeypatch.setenv("ECS_RK4CHAIN_MINB", "1")
        monkeypatch.setenv("ECS_RK4CHAIN_MAXB", "64")
    else:
        monkeypatch.setenv("ECS_RK4CHAIN_MAXB", "0")
    context.clear_cache()
    try:
        pd = E.make_param_dict(n, 1 / 50, 1 / 50, forcing="kolmogorov+")
        f = torch.as_tensor(np.fft.rfft2(np.stack([initial_condition(80 + b, n, amp=3.0) for b in range(B)])),
                            device="cuda")
        ctx = context.get_context(pd, n, torch.float64, B)
        torch.cuda.synchronize()
        c0 = ctx.lib.ecs_launch_count(ctx.handle)
        out = E.lawson_rk4(f, 0.004 * steps, steps, pd).cpu().clone()
        torch.cuda.synchronize()
        # objective_RPO in Lawson_RK4 mode shoots through the same stepping
        pdo = E.make_param_dict(n, 1 / 50, 1 / 50, forcing="kolmogorov+", num_checkpoints=2, ministeps=steps,
                                shift_reflect_ny=1, rot=False)
        obj = E.objective_RPO({"fields": torch.as_tensor(initial_condition(5, n), device="cuda"), "T": 0.1,
                               "sx": 0.3}, pdo, "Lawson_RK4")
        return out, obj["fields"].cpu().clone(), ctx.lib.ecs_launch_count(ctx.handle) - c0
    finally:
        monkeypatch.undo()
        context.clear_cache()


@pytest.mark.parametrize("n,B,steps", RK4_CASES)
def test_rk4_chain_equals_launch_per_stage(cuda, monkeypatch, n, B, steps):
    """Lawson-RK4 stepping as one cluster-resident launch (k_rk4_chain) equals
    the launch-per-stage stepping (graphs of k_row_rhs / k_col_rk4) bit for bit."""
    want, want_obj, per_stage = _rk4(n, B, steps, monkeypatch, chain=False)
    for v in [(8, 1, 0), (8, 0, 0), (16, 1, 0), (16, 0, 0)]:
        got, got_obj, chained = _rk4(n, B, steps, monkeypatch, chain=True, variant=v)
        assert torch.equal(got, want), v
        assert torch.equal(got_obj, want_obj), v
        assert chained < per_stage


def test_default_batch_ranges(cuda, monkeypatch):
    """With no switches set, one tangent at 128^2 runs through the chain (a few
    launches) and 64 tangents through the launch-per-pass sweep (the chain's
    clusters would not all fit on the device at once)."""
    for k in ("ECS_CHAIN_MINB", "ECS_CHAIN_MAXB", "ECS_CHAIN_WARPS", "ECS_CHAIN_DSMEM", "ECS_CHAIN_DSLOTS", "ECS_REGEN_ITEMS"):
        monkeypatch.delenv(k, raising=False)
    n, T = 128, 0.15
    pd = E.make_param_dict(n, 1 / 50, 1 / 50, forcing="kolmogorov+", shift_reflect_ny=1, rot=False,
                           adaptive_dict={"atol": 1e-8, "checkpoints": 4, "max_steps_per_checkpoint": 64})
    prim = {"fields": torch.as_tensor(initial_condition(4, n, amp=2.0), device="cuda"), "T": T, "sx": 0.2}
    context.clear_cache()
    try:
        counts = {}
        for B in (1, 64):
            du = np.stack([initial_condition(60 + i, n) * 0.1 for i in range(B)])
            tan = {"fields": torch.as_tensor(du, device="cuda"), "T": torch.zeros(B, dtype=torch.float64),
                   "sx": torch.zeros(B, dtype=torch.float64)}
            obj = E.Objective(pd, "Lawson_RK43")
            obj.linearize(prim, force=True, batch=B)
            ctx = context.get_context(pd, n, torch.float64, B)
            torch.cuda.synchronize()
            c0 = ctx.lib.ecs_launch_count(ctx.handle)
            obj.jvp(prim, tan)
            torch.cuda.synchronize()
            counts[B] = (ctx.lib.ecs_launch_count(ctx.handle) - c0, obj.last_info["accepted"])
        assert counts[1][0] < 20, counts
        assert counts[64][0] > 4 * counts[64][1], counts
    finally:
        context.clear_cache()


RK43_CASES = [   # (n, B, T, atol, amp, seed)
    (64, 1, 0.3, 1e-6, 6.0, 4),
    (64, 3, 0.3, 1e-6, 6.0, 4),
    (128, 2, 0.2, 1e-8, 2.0, 4),
    (128, 1, 0.5, 1e-8, 2.0, 0),   # the 128^2 matvec workload's trajectory: rejected attempts
]


def _rk43(n, B, T, atol, amp, seed, monkeypatch, chain, w=0):
    monkeypatch.setenv("ECS_CHAIN_MAXB", "0")   # the tangent sweep launched per pass in both runs
    if chain:
        monkeypatch.setenv("ECS_RK43CHAIN_MINB", "1")
        monkeypatch.setenv("ECS_RK43CHAIN_MAXB", "64")
        monkeypatch.setenv("ECS_CHAIN_WARPS", str(w))
    else:
        monkeypatch.setenv("ECS_RK43CHAIN_MAXB", "0")
    context.clear_cache()
    try:
        cap = (64, 64) if seed == 0 else (4, 64)
        pd = E.make_param_dict(n, 1 / 50, 1 / 50, forcing="kolmogorov+", shift_reflect_ny=1, rot=False,
                               adaptive_dict={"atol": atol, "checkpoints": cap[0], "max_steps_per_checkpoint": cap[1]})
        fields = torch.as_tensor(np.stack([initial_condition(seed + i, n, amp=amp) for i in range(B)]), device="cuda")
        batch = E.objective_RPO({"fields": fields, "T": torch.linspace(T, 1.2 * T, B, dtype=torch.float64),
                                 "sx": 0.2}, pd, "Lawson_RK43")["fields"].cpu().clone()
        # the recorded linearisation of candidate 0 and a JVP through it (launched per pass)
        prim = {"fields": fields[0].contiguous(), "T": T, "sx": 0.2}
        obj = E.Objective(pd, "Lawson_RK43")
        obj.linearize(prim, force=True, batch=1)
        info = dict(obj.last_info)
        du = torch.as_tensor(initial_condition(70, n) * 0.1, device="cuda")[None]
        jv = obj.jvp(prim, {"fields": du, "T": torch.tensor([0.3], dtype=torch.float64),
                            "sx": torch.tensor([-0.2], dtype=torch.float64)})
        return batch, info, {k: v.detach().cpu().clone() for k, v in jv.items()}
    finally:
        monkeypatch.undo()
        context.clear_cache()


@pytest.mark.parametrize("n,B,T,atol,amp,seed", RK43_CASES)
def test_rk43_chain_equals_launch_per_stage(cuda, monkeypatch, n, B, T, atol, amp, seed):
    """The adaptive Lawson-RK4(3) solve as one cluster-resident launch
    (k_rk43_chain: attempts, error norm and accept/reject decision on the
    device) equals the per-stage launches (k_col_rk43 / k_row_rhs / k_row_err)
    bit for bit: the batched objective, the step statistics and the recorded
    trajectory (through a JVP at the linearisation), with either CTA shape."""
    want, want_info, want_jv = _rk43(n, B, T, atol, amp, seed, monkeypatch, chain=False)
    for w in (8, 16):
        got, info, jv = _rk43(n, B, T, atol, amp, seed, monkeypatch, chain=True, w=w)
        assert torch.equal(got, want), w
        assert info == want_info, w
        for k in ("fields", "T", "sx"):
            assert torch.equal(jv[k], want_jv[k]), (k, w)
    if seed == 0:
        assert want_info["rejected"] > 0, want_info


def test_fp32_chains_equal_launch_per_pass(cuda, monkeypatch):
    """FP32 (the precision mode's stepping and JVPs) through the chains: Lawson-RK4
    stepping and a batch-1 adaptive JVP at n = 64 equal the per-pass launches bit
    for bit."""
    n = 64

    def run(chain):
        monkeypatch.setenv("ECS_CHAIN_MAXB", "64" if chain else "0")
        monkeypatch.setenv("ECS_RK4CHAIN_MAXB", "64" if chain else "0")
        monkeypatch.setenv("ECS_RK43CHAIN_MAXB", "64" if chain else "0")
        context.clear_cache()
        try:
            pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", data_type=torch.float32,
                                   shift_reflect_ny=1, rot=False,
                                   adaptive_dict={"atol": 1e-5, "checkpoints": 4, "max_steps_per_checkpoint": 64})
            f = torch.as_tensor(np.fft.rfft2(np.stack([initial_condition(80 + b, n, amp=3.0) for b in range(2)])),
                                dtype=torch.complex64, device="cuda")
            stepped = E.lawson_rk4(f, 0.1, 20, pd).cpu().clone()
            prim = {"fields": torch.as_tensor(initial_condition(4, n, amp=4.0), dtype=torch.float32, device="cuda"),
                    "T": 0.3, "sx": 0.2}
            obj = E.Objective(pd, "Lawson_RK43")
            obj.linearize(prim, force=True, batch=1)
            du = torch.as_tensor(initial_condition(61, n) * 0.1, dtype=torch.float32, device="cuda")[None]
            jv = obj.jvp(prim, {"fields": du, "T": torch.tensor([0.4], dtype=torch.float64),
                                "sx": torch.tensor([0.1], dtype=torch.float64)})
            return stepped, {k: v.detach().cpu().clone() for k, v in jv.items()}, dict(obj.last_info)
        finally:
            monkeypatch.undo()
            context.clear_cache()

    want = run(False)
    got = run(True)
    assert torch.equal(got[0], want[0])
    for k in ("fields", "T", "sx"):
        assert torch.equal(got[1][k], want[1][k]), k
    assert got[2] == want[2]
