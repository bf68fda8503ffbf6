"""Change of resolution of a state file (jax_scripts/upscale_state.py): the
library's change_resolution / upscale_state against the oracle's numpy
restatement, and the restatement's own properties (band-limited fields survive
up- and down-sampling exactly; the mean square is kept).  Tolerance 1e-12."""
import numpy as np
import torch

import oracle as O
import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import dictionaryIO
from ecs_mhd_2d_b200.synthetic import initial_condition


def test_oracle_round_trip_and_mean_square():
    u = initial_condition(5, 64)              # band-limited (|k| <= 8), no Nyquist content
    up = O.change_resolution(u, 128)
    back = O.change_resolution(up, 64)
    assert np.abs(back - u).max() <= 1e-12 * np.abs(u).max()
    assert abs(np.mean(up ** 2) - np.mean(u ** 2)) <= 1e-12 * np.mean(u ** 2)


def test_change_resolution_matches_oracle():
    rng = np.random.default_rng(3)
    for m, n in ((64, 128), (128, 256), (128, 64)):
        f = rng.standard_normal((2, m, m))
        got = dictionaryIO.change_resolution(torch.as_tensor(f), n).numpy()
        want = O.change_resolution(f, n)
        assert got.shape == (2, n, n)
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_upscale_state_round_trip(tmp_path):
    n = 64
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov", num_checkpoints=4, ministeps=8,
                           forcing_str="lambda x,y : -4*jnp.cos(4*y)")
    x = {"fields": torch.as_tensor(initial_condition(2, n)), "T": 1.5, "sx": 0.2}
    inp, par = dictionaryIO.upscale_state(x, pd, 128)
    assert inp["fields"].shape == (2, 128, 128) and par["x"].shape[-1] == 128
    assert inp["T"] == 1.5 and par["num_checkpoints"] == 4
    # the -4 cos(4y) forcing resampled equals the forcing built at n = 128
    assert torch.allclose(par["forcing"].cpu(), E.make_param_dict(128, 1 / 40, 1 / 40, forcing="kolmogorov")["forcing"].cpu(),
                          atol=1e-12)
    path = str(tmp_path / "up.npz")
    dictionaryIO.save_dicts(path, inp, par)
    inp2, par2 = dictionaryIO.load_dicts(path)
    assert np.allclose(inp2["fields"].numpy(), inp["fields"].numpy(), rtol=0, atol=0)
