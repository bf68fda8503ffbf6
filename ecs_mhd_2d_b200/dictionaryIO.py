"""State + parameter files in the reference's .npz format
(reference: jax_scripts/lib/dictionaryIO.py:11-78).

A file holds the input dict ("fields", "T", "sx") and the parameter dict
(nu, eta, b0, forcing_str, steps, ministeps, num_checkpoints, shift_reflect_ny,
rot, ...) with two key lists, "input_keys" and "param_keys".
"""

from __future__ import annotations

import ast
import math

import numpy as np
import torch

from .mhd import construct_domain, PI_LITERAL

GRID_KEYS = ["x", "y", "kx", "ky", "mask", "to_u", "to_v", "inv_lap", "forcing"]


def _np(v):
    if isinstance(v, torch.Tensor):
        return v.detach().cpu().numpy()
    return np.array(v)


def save_dicts(filename, input_dict, param_dict):
    """Merge both dicts with their key lists and np.savez them (dictionaryIO.py:11-27)."""
    combined = dict(input_dict)
    combined.update(param_dict)
    combined["input_keys"] = list(input_dict.keys())
    combined["param_keys"] = list(param_dict.keys())
    np.savez(filename, **{k: _np(v) for k, v in combined.items()})


def load_dicts(filename, device=None):
    """(input_dict, param_dict) from a file (dictionaryIO.py:30-48); numeric
    arrays become torch tensors (on `device` if given)."""
    loaded = np.load(filename, allow_pickle=True)

    def conv(val):
        if isinstance(val, np.ndarray) and np.issubdtype(val.dtype, np.number):
            t = torch.as_tensor(val)
            return t.to(device) if device is not None else t
        return val.item() if getattr(val, "shape", None) == () else val

    inp = {k: conv(loaded[k]) for k in loaded["input_keys"]}
    par = {k: conv(loaded[k]) for k in loaded["param_keys"]}
    return inp, par


def inspect_dict(d):
    """One line per key: shape, dtype and size in KB of array values, the type
    otherwise (inspect_dict of jax_scripts/test_solution_file_structure.py:17-25,
    returned as a list of lines instead of printed)."""
    lines = []
    for key, value in d.items():
        if isinstance(value, torch.Tensor):
            value = value.detach().cpu().numpy()
        if hasattr(value, "size") and hasattr(value, "dtype"):
            kb = value.size * value.dtype.itemsize / 1024
            lines.append(f"Key: {key}, shape: {value.shape}, dtype: {value.dtype}, size: {kb:.2f} KB")
        else:
            lines.append(f"Key: {key}, type: {type(value)}, size: unknown")
    return lines


def describe_file(filename):
    """The two sections that test_solution_file_structure.py:27-31 prints for a
    state file: "input_dict:" and "param_dict:" with inspect_dict's lines."""
    inp, par = load_dicts(filename)
    inp = {k: (v.numpy() if isinstance(v, torch.Tensor) else v) for k, v in inp.items()}
    par = {k: (v.numpy() if isinstance(v, torch.Tensor) else v) for k, v in par.items()}
    return "\n".join(["input_dict:"] + inspect_dict(inp) + ["", "param_dict:"] + inspect_dict(par))


def remove_grid_information(param_dict):
    """Drop the grid tensors before saving (dictionaryIO.py:52-60)."""
    pd = dict(param_dict)
    for key in GRID_KEYS:
        pd.pop(key, None)
    return pd


_FORCING_FUNCS = {"cos": np.cos, "sin": np.sin, "exp": np.exp, "tanh": np.tanh, "sqrt": np.sqrt,
                  "cosh": np.cosh, "sinh": np.sinh, "abs": np.abs}
_FORCING_CONSTS = {"pi": math.pi}
_FORCING_BINOPS = {ast.Add: np.add, ast.Sub: np.subtract, ast.Mult: np.multiply, ast.Div: np.divide,
                   ast.Pow: np.power}


def _forcing_eval(node, env):
    """Evaluate one node of a forcing expression: numbers, the two coordinates,
    + - * / **, unary minus, and jnp./np. math functions and pi; anything else
    is refused."""
    if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)) and not isinstance(node.value, bool):
        return float(node.value)
    if isinstance(node, ast.Name) and node.id in env:
        return env[node.id]
    if isinstance(node, ast.BinOp) and type(node.op) in _FORCING_BINOPS:
        return _FORCING_BINOPS[type(node.op)](_forcing_eval(node.left, env), _forcing_eval(node.right, env))
    if isinstance(node, ast.UnaryOp) and isinstance(node.op, (ast.USub, ast.UAdd)):
        v = _forcing_eval(node.operand, env)
        return -v if isinstance(node.op, ast.USub) else v
    if (isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name) and node.value.id in ("jnp", "np")
            and node.attr in _FORCING_CONSTS):
        return _FORCING_CONSTS[node.attr]
    if (isinstance(node, ast.Call) and isinstance(node.func, ast.Attribute) and isinstance(node.func.value, ast.Name)
            and node.func.value.id in ("jnp", "np") and node.func.attr in _FORCING_FUNCS
            and len(node.args) == 1 and not node.keywords):
        return _FORCING_FUNCS[node.func.attr](_forcing_eval(node.args[0], env))
    raise ValueError(f"forcing_str: unsupported expression {ast.dump(node)[:80]}")


def forcing_from_string(forcing_str, n):
    """The reference's forcing string, e.g. 'lambda x,y : -4*jnp.cos(4*y)'
    (jax_scripts/lib/dictionaryIO.py:74 evaluates it), on the grid of
    construct_domain.  The string is parsed, not executed: a lambda of two
    arguments whose body uses numbers, the arguments, + - * / **, and the
    jnp./np. functions cos sin exp tanh sqrt cosh sinh abs and the constant pi."""
    grid = np.arange(n, dtype=np.float64) / n * 2 * PI_LITERAL
    x, y = np.meshgrid(grid, grid, indexing="ij")
    try:
        tree = ast.parse(str(forcing_str).strip(), mode="eval")
    except SyntaxError as ex:
        raise ValueError(f"forcing_str: not an expression: {forcing_str!r}") from ex
    lam = tree.body
    if (not isinstance(lam, ast.Lambda) or len(lam.args.args) != 2 or lam.args.vararg or lam.args.kwarg
            or lam.args.kwonlyargs or lam.args.defaults or lam.args.posonlyargs):
        raise ValueError(f"forcing_str: expected 'lambda x,y : <expression>', got {forcing_str!r}")
    names = [a.arg for a in lam.args.args]
    val = _forcing_eval(lam.body, {names[0]: x, names[1]: y})
    return np.broadcast_to(np.asarray(val, dtype=np.float64), (n, n)).copy()


def recompute_grid_information(input_dict, param_dict):
    """Inverse of remove_grid_information (dictionaryIO.py:64-78)."""
    f = input_dict["fields"]
    n = f.shape[-1]
    dt = f.dtype if isinstance(f, torch.Tensor) else torch.float64
    param_dict.update(construct_domain(n, dt))
    fr = forcing_from_string(param_dict["forcing_str"], n)
    param_dict["forcing"] = torch.as_tensor(fr, dtype=dt, device=param_dict["x"].device)
    b0 = param_dict.get("b0", [0.0, 0.1])
    param_dict["b0"] = [float(b0[0]), float(b0[1])]
    return param_dict


def change_resolution(f, n):
    """A real field [..., m, m] resampled to [..., n, n] spectrally
    (jax_scripts/upscale_state.py:29-47): fft2, the four corner blocks of
    min(m, n)//2 wavenumbers copied (the Nyquist line is dropped), ifft2 scaled
    by (n/m)^2, real part.  Runs on the tensor's device."""
    f = torch.as_tensor(f)
    m = f.shape[-1]
    F = torch.fft.fft2(f.to(torch.float64))
    F2 = torch.zeros(tuple(f.shape[:-2]) + (n, n), dtype=torch.complex128, device=f.device)
    m2 = min(m, n) // 2
    F2[..., :m2, :m2] = F[..., :m2, :m2]
    F2[..., n - m2:, :m2] = F[..., m - m2:, :m2]
    F2[..., :m2, n - m2:] = F[..., :m2, m - m2:]
    F2[..., n - m2:, n - m2:] = F[..., m - m2:, m - m2:]
    return (torch.fft.ifft2(F2) * (n / m) ** 2).real


def upscale_state(input_dict, param_dict, n):
    """A state and its parameters at resolution n (jax_scripts/upscale_state.py:48-63):
    both field channels and the forcing resampled by change_resolution, the grid
    tables rebuilt for n; T, sx and the other parameters unchanged.  Returns
    new (input_dict, param_dict); save_dicts writes them in the reference's
    format (the forcing is stored as its forcing_str, as the reference does)."""
    fields = torch.as_tensor(input_dict["fields"])
    inp = dict(input_dict)
    inp["fields"] = change_resolution(fields, n).to(fields.dtype)
    par = dict(param_dict)
    dt = fields.dtype if fields.is_floating_point() else torch.float64
    par.update(construct_domain(n, dt))
    if "forcing" in param_dict:
        fr = change_resolution(torch.as_tensor(param_dict["forcing"]), n)
        par["forcing"] = fr.to(dtype=dt, device=par["x"].device)
    return inp, par
