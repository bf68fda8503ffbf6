"""DNS data generation (jax_scripts/generate_turbulence.py) on the GPU against
the oracle's Lawson-RK6 and a direct numpy recurrence matrix; the saved file
has the reference's layout.  Tolerance 1e-12 relative (FP64, short runs)."""
import numpy as np
import pytest
import torch

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import dictionaryIO, turbulence
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_generate_turbulence_matches_oracle(cuda, tmp_path):
    n, dt, ms, steps, tr = 64, 1 / 256, 8, 4, 16
    path = str(tmp_path / "turb.npz")
    fs, dist, pd = turbulence.generate_turbulence(n=n, dt=dt, ministeps=ms, steps=steps, transient_steps=tr,
                                                  seed=3, path=path)
    # oracle: the same initial data, transient and snapshots
    opd = O.make_param_dict(n, 1 / 40, 1 / 40, b0=(0.0, 0.3), forcing="kolmogorov")
    f = np.fft.rfft2(10.0 * np.random.default_rng(3).standard_normal((2, n, n))) * opd["mask"]
    v = lambda x: O.state_vel(x, opd, False)
    L = O.dissipation(opd)
    f = O.lawson_rk6(f, dt * tr, tr, v, L, opd["mask"])
    want = []
    for _ in range(steps):
        f = O.lawson_rk6(f, dt * ms, ms, v, L, opd["mask"])
        want.append(f)
    want = np.stack(want)
    got = fs.cpu().numpy()
    assert rel_l2(np.fft.irfft2(got, s=(n, n)), np.fft.irfft2(want, s=(n, n))) < 1e-12
    mag = np.abs(want).reshape(steps, -1)
    wd = np.sqrt(((mag[:, None, :] - mag[None, :, :]) ** 2).sum(-1))
    assert np.abs(dist.cpu().numpy() - wd).max() <= 1e-12 * wd.max()
    inp, par = dictionaryIO.load_dicts(path)
    assert set(inp) == {"fs", "dist"} and par["ministeps"] == ms and par["steps"] == steps


@pytest.mark.parametrize("mode", ["RK4", "TDRK4", "Lawson_RK6"])
def test_integrate_modes_keep_or_zero_outside_box(cuda, mode):
    """ecs_integrate on a full half spectrum: RK4 and TDRK4 keep the modes
    outside the box (masked right-hand side), Lawson_RK6 zeroes them; the box
    modes match the oracle's stepper."""
    n = 64
    opd = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+")
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+")
    f0 = np.fft.rfft2(np.random.default_rng(7).standard_normal((2, n, n)))
    t, steps = 0.05, 10
    got = E.integrate(torch.as_tensor(f0, device="cuda"), t, steps, pd, mode).cpu().numpy()
    if mode == "Lawson_RK6":
        want = O.lawson_rk6(f0, t, steps, lambda x: O.state_vel(x, opd, False), O.dissipation(opd), opd["mask"])
    elif mode == "RK4":
        want = O.rk4(f0, t, steps, lambda x: O.state_vel(x, opd, True))
    else:
        want = O.tdrk4(f0, t, steps, lambda x: O.state_vel(x, opd, True),
                       lambda x, k: O.state_vel_jvp(x, k, opd, True))
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)
