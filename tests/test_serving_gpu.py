"""Continuous-batching server: every request's result is the same alone and in
the mix (the bound written is 1e-12: batched matvecs take the primal fields
from another pass of the same arithmetic than a single-candidate call),
requests that arrive while others run are admitted into free slots, the slot
pool keeps serving requests of different horizons side by side, and matvec or
gradient requests that queue up together are swept as one batch."""
import numpy as np
import pytest
import torch

import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import serving
from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12


def alone(req):
    pd = serving._param_dict(req, req.dtype)
    x = {"fields": torch.as_tensor(req.fields, dtype=req.dtype, device="cuda"), "T": req.T, "sx": req.sx}
    if req.kind == "forward" and req.mode == "Lawson_RK4":
        out = E.objective_RPO(x, pd, "Lawson_RK4")
        loss, _ = E.loss_RPO(x, pd, "Lawson_RK4")
        return {"fields": out["fields"], "loss": float(loss)}
    ctx = serving.C.Context(req.n, req.dtype, 1 / req.Re, 1 / req.Re, pd["b0"],
                            serving.C._forcing_key(pd["forcing"])[1], max_batch=1)
    return serving.run_adjoint_request(req, ctx, torch.cuda.current_stream())


def test_results_identical_alone_and_in_the_mix(cuda):
    reqs = serving.poisson_requests(14, rate=400.0, seed=3, ns=(64, 128), horizons=(64, 96, 160),
                                    Res=(40.0, 50.0), adaptive_fraction=0.3)
    assert {r.mode for r in reqs} == {"Lawson_RK4", "Lawson_RK43"}
    srv = serving.Server(hbm_budget=24 << 30, slots=4, chunk_steps=16, workers_per_group=2)
    res = srv.run(reqs)
    assert [r.rid for r in res] == list(range(len(reqs)))
    # requests overlapped: some were admitted before earlier ones finished
    assert any(res[i].t_admit < max(res[j].t_done for j in range(i)) for i in range(1, len(res)))
    for req, r in zip(reqs, res):
        a = alone(req)
        assert rel_l2(r.out["fields"].cpu().numpy(), a["fields"].cpu().numpy()) <= TOL, (req.kind, req.n)
        if "loss" in a:
            assert abs(r.out["loss"] - a["loss"]) <= TOL * abs(a["loss"])


def test_pool_mixes_horizons(cuda):
    """Slots with different step budgets finish at different times and a new
    request takes a freed slot while the others keep running."""
    from ecs_mhd_2d_b200.synthetic import initial_condition
    n = 64
    pool = serving.ForwardPool(n, torch.float64, 40.0, slots=2)
    mk = lambda rid, steps: serving.Request(rid, "forward", n, steps, 40.0, steps * 0.005, 0.1,
                                            initial_condition(rid, n))
    r0, r1, r2 = mk(0, 16), mk(1, 48), mk(2, 16)
    pool.admit(r0, 0.0)
    pool.admit(r1, 0.0)
    pool.advance(16)
    done = pool.harvest(lambda: 1.0)
    assert [d.rid for d in done] == [0]
    pool.admit(r2, 1.0)           # r1 is 16 steps into its 48
    pool.advance(16)
    done = pool.harvest(lambda: 2.0)
    assert [d.rid for d in done] == [2]
    pool.advance(16)
    done = pool.harvest(lambda: 3.0)
    assert [d.rid for d in done] == [1]
    a = alone(r1)
    assert rel_l2(done[0].out["fields"].cpu().numpy(), a["fields"].cpu().numpy()) <= TOL


@pytest.mark.parametrize("kind", ["matvec", "gradient"])
def test_burst_is_batched(cuda, kind):
    """Eight matvec (or gradient) requests of one group, of different horizons,
    arriving together: the batcher sweeps several of them in one ecs_jvp_multi
    (ecs_loss_grad_multi) call, and every result equals the request run alone."""
    reqs = serving.poisson_requests(8, rate=1e5, seed=11, ns=(64,), horizons=(64, 96, 128), Res=(40.0,),
                                    kinds=(kind,), adaptive_fraction=0.0)
    srv = serving.Server(hbm_budget=16 << 30, slots=8, chunk_steps=16, workers_per_group=1)
    res = srv.run(reqs)
    sweeps = [b.sweeps for b in srv.batchers.values()]
    assert len(sweeps) == 1 and sum(sweeps[0]) == 8 and max(sweeps[0]) > 1, sweeps
    for req, r in zip(reqs, res):
        a = alone(req)
        assert rel_l2(r.out["fields"].cpu().numpy(), a["fields"].cpu().numpy()) <= TOL
        assert abs(r.out["T"] - float(a["T"])) <= TOL * max(abs(float(a["T"])), 1.0)
        if kind == "gradient":
            assert abs(r.out["loss"] - a["loss"]) <= TOL * abs(a["loss"])
