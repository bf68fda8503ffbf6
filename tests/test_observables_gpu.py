"""Energy observables along an orbit (jax_scripts/projection.py): the device
TDRK4 steps and torch observables against the oracle's tdrk4 and numpy
restatement of compute_observables / laminar_flow, 1e-11 relative (FP64,
six steps)."""
import numpy as np
import pytest
import torch

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import observables
from ecs_mhd_2d_b200.synthetic import initial_condition

pytestmark = pytest.mark.gpu


def test_projection_matches_oracle(cuda):
    n, steps, T = 64, 6, 0.06
    u0 = initial_condition(4, n)
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, b0=(0.0, 0.1), forcing="kolmogorov", steps=steps)
    opd = O.make_param_dict(n, 1 / 40, 1 / 40, b0=(0.0, 0.1), forcing="kolmogorov")
    got = observables.projection({"fields": u0, "T": T, "sx": 0.0}, pd).cpu().numpy()
    v = lambda f: O.state_vel(f, opd, True)
    jac = lambda f, k: O.state_vel_jvp(f, k, opd, True)
    f = np.fft.rfft2(u0)
    want = np.zeros((2, steps))
    for i in range(steps):
        want[:, i] = O.compute_observables(f, opd)
        f = O.tdrk4(f, T / steps, 1, v, jac)
    want /= O.compute_observables(np.fft.rfft2(O.laminar_flow(opd)), opd).reshape(2, 1)
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()
