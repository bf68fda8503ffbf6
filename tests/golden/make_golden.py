"""Generate the committed golden fixtures under tests/golden/.

1. Reference solutions: a subset of the reference's converged states
   (solutions/Re40/*.npz, solutions/Re50/*.npz of mgolden30/ECS_MHD_2D) is copied
   with their parameters, together with the closure residual
   |g.Phi_T(u0) - u0| / |u0| that the oracle's Lawson-RK4 gives for ALL fifteen
   solutions (closure_lawson_rk4.json).  Small closure pins the oracle to the
   reference's physics: RHS, forcing sign, dissipation, symmetries.
2. Synthetic seeded cases at n=64 computed by the oracle (synthetic_n64.npz):
   state_vel, 64 Lawson-RK4 steps, objective and loss.
3. Closure of all fifteen reference solutions under each fixed-step mode
   (closure_modes.json: Lawson_RK4, TDRK4, RK4).  The reference does not store
   which integrator converged a solution; the mode that closes one to rounding
   level is the one it was converged with, which pins that mode's oracle.

4. The headline matvec at its full horizon (headline_jvp_n128.npz): the
   objective value and the JVP of tangent 0 of the benchmark's 64-tangent
   batch, at the benchmark's own workload (n=128 FP64, Re=50, Lawson_RK43 atol
   1e-8, T=4.6, sx=0.12, seed-0 amplitude-2 state), by torch.func.jvp of the
   oracle's torch form (minutes of CPU time, hence a fixture).

Run from the repository root:
    python tests/golden/make_golden.py /path/to/reference [modes]   (1-3: needs the reference checkout)
    python tests/golden/make_golden.py headline                      (4: the oracle only)
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

import oracle as O  # noqa: E402
from ecs_mhd_2d_b200.synthetic import initial_condition  # noqa: E402

KEEP = ["Re40/RPO5", "Re40/RPO6", "Re40/TW1", "Re40/EQ1", "Re50/RPO2"]
PARAM_KEYS = ["nu", "eta", "b0", "steps", "ministeps", "num_checkpoints", "shift_reflect_ny", "rot"]


def param_dict_from(d):
    n = d["fields"].shape[-1]
    return O.make_param_dict(n, float(d["nu"]), float(d["eta"]), b0=d["b0"],
                             num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
                             shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))


def solutions(ref):
    rec = {}
    for sub in ["Re40", "Re50"]:
        for fn in sorted(os.listdir(os.path.join(ref, "solutions", sub))):
            name = f"{sub}/{fn[:-4]}"
            d = np.load(os.path.join(ref, "solutions", sub, fn), allow_pickle=True)
            assert str(d["forcing_str"]) == "lambda x,y : -4*jnp.cos(4*y)"
            pd = param_dict_from(d)
            inp = {"fields": d["fields"], "T": float(d["T"]), "sx": float(d["sx"])}
            out = O.objective_RPO(inp, pd, "Lawson_RK4")
            r = float(np.linalg.norm(out["fields"]) / np.linalg.norm(d["fields"]))
            rec[name] = {"n": int(d["fields"].shape[-1]), "steps": int(d["steps"]), "closure": r,
                         "T": float(d["T"]), "sx": float(d["sx"])}
            print(name, rec[name], flush=True)
            if name in KEEP:
                np.savez_compressed(os.path.join(HERE, f"solution_{sub}_{fn[:-4]}.npz"),
                                    fields=d["fields"], T=d["T"], sx=d["sx"], closure=r,
                                    residual_norm=np.linalg.norm(out["fields"]),
                                    **{k: d[k] for k in PARAM_KEYS})
    with open(os.path.join(HERE, "closure_lawson_rk4.json"), "w") as f:
        json.dump(rec, f, indent=1, sort_keys=True)


def synthetic():
    n, seed = 64, 0
    u0 = initial_condition(seed, n)
    pd = O.make_param_dict(n, 1 / 40, 1 / 40, forcing="kolmogorov+", num_checkpoints=2, ministeps=32,
                           shift_reflect_ny=1, rot=True)
    f0 = np.fft.rfft2(u0)
    sv = O.state_vel(f0, pd, False)
    svd = O.state_vel(f0, pd, True)
    L = O.dissipation(pd)
    v_fn = lambda f: O.state_vel(f, pd, False)
    f64 = O.lawson_rk4(f0, 64 * 0.005, 64, v_fn, L, mask=pd["mask"])
    inp = {"fields": u0, "T": 0.32, "sx": 0.3}
    obj = O.objective_RPO(inp, pd, "Lawson_RK4")
    loss, _ = O.loss_RPO(inp, pd, "Lawson_RK4")
    np.savez_compressed(os.path.join(HERE, "synthetic_n64.npz"), u0=u0, seed=seed, nu=1 / 40, eta=1 / 40,
                        forcing_amp=4.0, state_vel=sv, state_vel_diss=svd, rk4_64=np.fft.irfft2(f64, s=(n, n)),
                        T=0.32, sx=0.3, num_checkpoints=2, ministeps=32, shift_reflect_ny=1, rot=True,
                        objective=obj["fields"], loss=loss)


def headline_jvp():
    import torch
    from torch.func import jvp
    from ecs_mhd_2d_b200.synthetic import unit_tangents
    torch.set_num_threads(os.cpu_count() or 1)
    n, T, sx, B = 128, 4.6, 0.12, 64
    ad = {"atol": 1e-8, "checkpoints": 64, "max_steps_per_checkpoint": 64}
    kw = dict(forcing="kolmogorov+", shift_reflect_ny=0, rot=False, adaptive_dict=ad)
    u0 = initial_condition(0, n, amp=2.0)
    t0 = unit_tangents(0, n, B)[0]
    _, _, info = O.mismatch_RPO({"fields": u0, "T": T, "sx": sx}, O.make_param_dict(n, 1 / 50, 1 / 50, **kw),
                                "Lawson_RK43")
    pdt = O.make_param_dict(n, 1 / 50, 1 / 50, xp=O.TORCH, **kw)
    f = lambda d: O.objective_RPO(d, pdt, "Lawson_RK43", xp=O.TORCH)
    prim = {"fields": torch.from_numpy(u0), "T": torch.tensor(T, dtype=torch.float64),
            "sx": torch.tensor(sx, dtype=torch.float64)}
    tan = {"fields": torch.from_numpy(np.ascontiguousarray(t0[1:-1].reshape(2, n, n))),
           "T": torch.tensor(t0[0], dtype=torch.float64), "sx": torch.tensor(t0[-1], dtype=torch.float64)}
    val, out = jvp(f, (prim,), (tan,))
    np.savez_compressed(os.path.join(HERE, "headline_jvp_n128.npz"), objective=val["fields"].numpy(),
                        jvp_fields=out["fields"].numpy(), jvp_T=out["T"].numpy(), jvp_sx=out["sx"].numpy(),
                        accepted=info["accepted"], rejected=info["rejected"], T=T, sx=sx, tangent_index=0)


def closure_by_mode(ref, modes=("Lawson_RK4", "TDRK4", "RK4")):
    rec = {}
    for sub in ["Re40", "Re50"]:
        for fn in sorted(os.listdir(os.path.join(ref, "solutions", sub))):
            name = f"{sub}/{fn[:-4]}"
            d = np.load(os.path.join(ref, "solutions", sub, fn), allow_pickle=True)
            pd = param_dict_from(d)
            inp = {"fields": d["fields"], "T": float(d["T"]), "sx": float(d["sx"])}
            rec[name] = {"n": int(d["fields"].shape[-1]), "steps": int(d["steps"])}
            for mode in modes:
                out = O.objective_RPO(inp, pd, mode)
                rec[name][mode] = float(np.linalg.norm(out["fields"]) / np.linalg.norm(d["fields"]))
            print(name, rec[name], flush=True)
    with open(os.path.join(HERE, "closure_modes.json"), "w") as f:
        json.dump(rec, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py (/path/to/reference [modes] | headline)")
    ref = sys.argv[1]
    if ref == "headline":
        headline_jvp()
    elif len(sys.argv) > 2 and sys.argv[2] == "modes":
        closure_by_mode(ref)
    else:
        synthetic()
        solutions(ref)
