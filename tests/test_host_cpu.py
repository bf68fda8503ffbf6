"""Host-side logic without a GPU: flat-vector order, state files, forcing
strings, line search, ADAM."""
import numpy as np
import torch

import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import dictionaryIO, drivers, utils


def test_flatten_order_matches_ravel_pytree():
    d = {"fields": torch.arange(8, dtype=torch.float64).reshape(2, 2, 2), "T": 5.0, "sx": -1.0}
    v = utils.flatten(d)
    assert v[0] == 5.0 and v[-1] == -1.0 and torch.equal(v[1:-1], torch.arange(8, dtype=torch.float64))
    back = utils.unflatten(v, 2)
    assert torch.equal(back["fields"], d["fields"]) and float(back["T"]) == 5.0


def test_forcing_string_of_the_reference_files():
    fr = dictionaryIO.forcing_from_string("lambda x,y : -4*jnp.cos(4*y)", 64)
    y = np.arange(64) / 64 * 2 * 3.14159265358979323846
    assert np.array_equal(fr, -4 * np.cos(4 * np.meshgrid(y, y, indexing="ij")[1]))


def test_forcing_string_is_parsed_not_executed():
    """Other arithmetic forms evaluate; anything beyond numbers, the two
    coordinates, + - * / ** and jnp./np. math is refused before it runs."""
    fr = dictionaryIO.forcing_from_string("lambda a, b: 2*jnp.sin(3*a)**2 - np.exp(-b/jnp.pi)", 16)
    g = np.arange(16) / 16 * 2 * 3.14159265358979323846
    x, y = np.meshgrid(g, g, indexing="ij")
    assert np.allclose(fr, 2 * np.sin(3 * x) ** 2 - np.exp(-y / np.pi), rtol=0, atol=1e-15)
    assert np.array_equal(dictionaryIO.forcing_from_string("lambda x,y: 3", 4), np.full((4, 4), 3.0))
    bad = ["__import__('os').system('true')", "lambda x,y: x.__class__", "lambda x,y: open('f')",
           "lambda x: x", "lambda x,y: jnp.linalg.norm(x)", "lambda x,y: [x]", "lambda x,y: jnp.cos(x, y)",
           "lambda x,y: True", "lambda x,y: 'a'"]
    for s in bad:
        try:
            dictionaryIO.forcing_from_string(s, 4)
        except ValueError:
            continue
        raise AssertionError(f"accepted {s!r}")


def test_save_load_round_trip(tmp_path):
    inp = {"fields": torch.randn(2, 64, 64, dtype=torch.float64), "T": torch.tensor(4.6, dtype=torch.float64),
           "sx": torch.tensor(0.1, dtype=torch.float64)}
    par = {"nu": 0.025, "eta": 0.025, "b0": [0.0, 0.1], "forcing_str": "lambda x,y : -4*jnp.cos(4*y)",
           "steps": 640, "ministeps": 32, "num_checkpoints": 20, "shift_reflect_ny": 1, "rot": True}
    fn = str(tmp_path / "state.npz")
    dictionaryIO.save_dicts(fn, inp, par)
    i2, p2 = dictionaryIO.load_dicts(fn)
    assert torch.equal(i2["fields"], inp["fields"]) and float(i2["T"]) == 4.6
    assert p2["forcing_str"] == par["forcing_str"] and int(p2["steps"]) == 640 and bool(p2["rot"])
    p2 = dictionaryIO.recompute_grid_information(i2, p2)
    assert p2["mask"].shape == (64, 33) and p2["forcing"].shape == (64, 64)
    assert "forcing" not in dictionaryIO.remove_grid_information(p2)


def test_describe_state_file(tmp_path):
    inp = {"fields": torch.zeros(2, 64, 64, dtype=torch.float64), "T": torch.tensor(4.6, dtype=torch.float64),
           "sx": torch.tensor(0.1, dtype=torch.float64)}
    par = {"nu": 0.025, "forcing_str": "lambda x,y : -4*jnp.cos(4*y)", "steps": 640}
    fn = str(tmp_path / "state.npz")
    dictionaryIO.save_dicts(fn, inp, par)
    text = dictionaryIO.describe_file(fn).splitlines()
    assert text[0] == "input_dict:" and text[4] == "" and text[5] == "param_dict:"
    assert text[1] == "Key: fields, shape: (2, 64, 64), dtype: float64, size: 64.00 KB"
    assert text[2] == "Key: T, shape: (), dtype: float64, size: 0.01 KB"
    assert text[7].startswith("Key: forcing_str, ") and len(text) == 9


def test_line_search_halves_until_improvement():
    target = torch.tensor([1.0, 2.0, 3.0], dtype=torch.float64)
    obj = lambda d: {"fields": d["fields"] - target.reshape(1, 1, 3)[..., :1].expand(2, 1, 1), "T": d["T"] * 0,
                     "sx": d["sx"] * 0}
    x = torch.zeros(4, dtype=torch.float64)
    step = torch.tensor([0.0, -10.0, -10.0, 0.0], dtype=torch.float64)   # overshoots: needs damping
    f_vec = utils.flatten(obj(utils.unflatten(x, 1)))
    unrav = lambda v: {"T": v[0], "fields": v[1:-1].reshape(2, 1, 1), "sx": v[-1]}
    x2, damp = utils.line_search_unravel(x, step, obj, unrav, f_vec)
    assert damp < 1.0 and torch.linalg.norm(utils.flatten(obj(unrav(x2)))) < torch.linalg.norm(f_vec)


def test_adam_matches_reference_formula():
    p = {"a": torch.tensor([1.0, -2.0], dtype=torch.float64)}
    g = {"a": torch.tensor([0.5, 0.25], dtype=torch.float64)}
    m, v = drivers.init_adam(p)
    p1, m, v = drivers.adam_update(p, g, m, v, 1, lr=1e-2, eps=1e-6)
    # first step: m_hat = g, v_hat = g^2 -> p - lr * g / (|g| + eps)
    want = p["a"] - 1e-2 * g["a"] / (g["a"].abs() + 1e-6)
    assert torch.allclose(p1["a"], want, rtol=0, atol=1e-15)
