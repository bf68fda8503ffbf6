"""Host logic of the serving workload: the seeded Poisson request stream and
the split of a horizon into checkpoint segments (no device calls)."""
import numpy as np
import torch

from ecs_mhd_2d_b200 import serving


def test_poisson_stream_is_seeded_and_mixed():
    a = serving.poisson_requests(300, rate=40.0, seed=7)
    b = serving.poisson_requests(300, rate=40.0, seed=7)
    c = serving.poisson_requests(300, rate=40.0, seed=8)
    assert [(r.kind, r.n, r.steps, r.arrival) for r in a] == [(r.kind, r.n, r.steps, r.arrival) for r in b]
    assert all(np.array_equal(x.fields, y.fields) for x, y in zip(a, b))
    assert [r.arrival for r in a] != [r.arrival for r in c]
    t = np.array([r.arrival for r in a])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 40.0) < 0.25 / 40.0           # exponential gaps of mean 1/rate
    assert {r.kind for r in a} == {"forward", "matvec", "gradient"}
    assert {r.n for r in a} == {64, 128, 256} and {r.steps for r in a} == {256, 512, 1024, 2048}
    for r in a:
        assert r.fields.shape == (2, r.n, r.n)
        assert r.dtype == (torch.float32 if r.n == 256 else torch.float64)
        assert abs(r.T - r.steps * 0.005 * 64 / r.n) < 1e-12
        assert (r.tangent is not None) == (r.kind == "matvec")
        if r.kind == "matvec":
            assert r.tangent.shape == (2 * r.n * r.n + 2,) and abs(np.linalg.norm(r.tangent) - 1) < 1e-12
        assert r.mode in ("Lawson_RK4", "Lawson_RK43")
        if r.mode == "Lawson_RK43":
            assert r.dtype == torch.float64
    assert {r.mode for r in a} == {"Lawson_RK4", "Lawson_RK43"}


def test_checkpoint_segments():
    for steps in (256, 512, 1024, 2048, 1088, 100):
        nc, ms = serving._nc_ms(steps)
        assert nc * ms == steps
        assert ms == (32 if steps % 32 == 0 else steps)
