"""Headline benchmark: Newton-GMRES matvec batch at 128^2 in FP64.

Workload (one bench step): linearise objective_RPO of mgolden30/ECS_MHD_2D in
Lawson_RK43 mode at a seeded base point (n=128, Re=Rm=50, Kolmogorov forcing
+4cos(4y), b0=[0,0.1], T=4.6, sx=0.12, atol=1e-8, cap 64x64 attempts) and push a
batch of 64 seeded unit-norm tangents [T, fields, sx] through the hand-written
tangent kernels: 64 JVP matvecs (jax_scripts/newton.py:165; jax.jvp at
jax_scripts/lib/utils.py:108).  The primal adaptive solve with its trajectory
record is inside every timed step; it runs through ecs_linearize_jvp, which
overlaps the batch-1 primal with the tangent sweep as jax.jvp computes both.
`config.phase_ms` reports the two halves run separately.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs an independent replica on its own GPU
(no data-path collective; weak scaling); the step time is the max over ranks.
`--impl reference` times the reference algorithm's CPU restatement (the oracle,
torch-CPU forward-mode AD as jax.jvp) on the host cores for a bounded sample of
the same workload; only rank 0 runs it.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 128
BATCH = 64
RE = 50.0
T0, SX0 = 4.6, 0.12
ATOL = 1e-8
CAP = (64, 64)
IC_SEED, IC_AMP = 0, 2.0
METRIC = "GMRES matvecs/s (JVP of objective_RPO, Lawson_RK43 atol 1e-8, T=4.6) at 128^2 FP64"
UNIT = "matvec/s"


def workload_config():
    """The workload both arms run (identical in both lines; measured results go
    to other keys)."""
    return {"workload": "newton_gmres_matvec_batch", "n": N, "dtype": "f64", "Re": RE, "forcing": "+4cos(4y)",
            "b0": [0.0, 0.1], "T": T0, "sx": SX0, "mode": "Lawson_RK43", "atol": ATOL,
            "checkpoints_x_max_steps": list(CAP), "krylov_batch": BATCH, "ic": f"seed {IC_SEED}, amp {IC_AMP}",
            "tangents": f"unit_tangents(seed rank, n, {BATCH})",
            "l2": "device arm: flushed (256 MiB write) before every timed step", "parallelism": "replicas"}


def param_dict(E):
    ad = {"atol": ATOL, "checkpoints": CAP[0], "max_steps_per_checkpoint": CAP[1]}
    return E.make_param_dict(N, 1 / RE, 1 / RE, forcing="kolmogorov+", shift_reflect_ny=0, rot=False,
                             adaptive_dict=ad)


def max_over_ranks(x, world, device):
    """The maximum of a per-rank time over all ranks: replicas are timed
    independently and the job takes as long as its slowest rank."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def whole_job_rate(world, units_per_rank, t_max_s):
    """Units processed by all ranks per second of the slowest rank (weak scaling)."""
    return world * units_per_rank / t_max_s


def host_inputs(seed):
    from ecs_mhd_2d_b200.synthetic import initial_condition, unit_tangents
    u0 = initial_condition(IC_SEED + seed, N, amp=IC_AMP)
    tv = unit_tangents(seed, N, BATCH)
    return u0, tv


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.samples, self._stop, self._t = index, [], threading.Event(), None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def _timed(torch, flush, fn):
    fn()
    flush.zero_()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3, out


def secondary_workloads(E, torch, dev, flush):
    """One timed repetition (after a warm-up) of the other measurement configs:
    config 0 (n=64 FP64 Lawson-RK4, dt=0.005, 1024 steps, seeds 0..7),
    config 2 (n=128 FP64 adjoint gradient, 1088 steps, T=4.26, checkpoints every 32),
    config 3 (n=256 FP32 stepping and JVP, 2048 steps, T=4.6; FP64 residual check)."""
    from ecs_mhd_2d_b200.synthetic import initial_condition, unit_tangents
    out = {}
    # config 0
    n0 = 64
    pd0 = E.make_param_dict(n0, 1 / 40, 1 / 40, forcing="kolmogorov+")
    f0 = torch.as_tensor(np.fft.rfft2(np.stack([initial_condition(s, n0) for s in range(8)])), device=dev)
    t, fT = _timed(torch, flush, lambda: E.lawson_rk4(f0, 1024 * 0.005, 1024, pd0))
    out["config0_rk4_n64_f64"] = {"state_steps_per_s": 8 * 1024 / t, "seconds": t, "batch": 8, "steps": 1024,
                                  "finite": bool(torch.isfinite(fT).all())}
    # config 2
    n2 = 128
    pd2 = E.make_param_dict(n2, 1 / 40, 1 / 40, forcing="kolmogorov+", num_checkpoints=34, ministeps=32,
                            shift_reflect_ny=0, rot=False, ckpt_every=32)
    x2 = {"fields": torch.as_tensor(initial_condition(2, n2, amp=IC_AMP), device=dev), "T": 4.26, "sx": 0.1}
    t, (lg, g) = _timed(torch, flush, lambda: E.loss_and_grad(x2, pd2, "Lawson_RK4", normalized=True))
    out["config2_gradient_n128_f64"] = {"gradients_per_s": 1.0 / t, "seconds": t, "steps": 1088,
                                        "ckpt_every": 32, "loss": float(lg[0])}
    # config 3
    n3 = 256
    pd3_64 = E.make_param_dict(n3, 1 / 50, 1 / 50, forcing="kolmogorov+", num_checkpoints=64, ministeps=32,
                               shift_reflect_ny=0, rot=False)
    pd3_32 = E.make_param_dict(n3, 1 / 50, 1 / 50, forcing="kolmogorov+", num_checkpoints=64, ministeps=32,
                               shift_reflect_ny=0, rot=False, data_type=torch.float32)
    u3 = initial_condition(3, n3, amp=IC_AMP)
    x64 = {"fields": torch.as_tensor(u3, device=dev), "T": 4.6, "sx": 0.12}
    x32 = {"fields": torch.as_tensor(u3, dtype=torch.float32, device=dev), "T": 4.6, "sx": 0.12}
    t32, o32 = _timed(torch, flush, lambda: E.objective_RPO(x32, pd3_32, "Lawson_RK4"))
    t64, o64 = _timed(torch, flush, lambda: E.objective_RPO(x64, pd3_64, "Lawson_RK4"))
    err = float(torch.linalg.norm(o32["fields"].double() - o64["fields"]) / torch.linalg.norm(o64["fields"]))
    obj32 = E.Objective(pd3_32, "Lawson_RK4")
    obj64 = E.Objective(pd3_64, "Lawson_RK4")
    Bt = 64
    tv = unit_tangents(5, n3, Bt)
    tan64 = {"fields": torch.as_tensor(tv[:, 1:-1].reshape(Bt, 2, n3, n3), device=dev),
             "T": torch.as_tensor(tv[:, 0]), "sx": torch.as_tensor(tv[:, -1])}
    tan32 = {"fields": tan64["fields"].float(), "T": tan64["T"], "sx": tan64["sx"]}
    tj32, o32 = _timed(torch, flush, lambda: obj32.linearize_jvp(x32, tan32)[1])
    tj64, o64 = _timed(torch, flush, lambda: obj64.linearize_jvp(x64, tan64)[1])
    terr = float(torch.linalg.norm(o32["fields"].double() - o64["fields"]) / torch.linalg.norm(o64["fields"]))
    # plain FP64: one tangent at a time at the fixed linearisation, as sequential GMRES issues them
    obj64.linearize(x64, force=True, batch=1)
    t1 = {"fields": tan64["fields"][:1].contiguous(), "T": tan64["T"][:1], "sx": tan64["sx"][:1]}
    tb1, _ = _timed(torch, flush, lambda: obj64.jvp(x64, t1))
    # batched FP32 stepping: 64 states, 256 Lawson-RK4 steps
    pd3s = E.make_param_dict(n3, 1 / 50, 1 / 50, forcing="kolmogorov+", data_type=torch.float32)
    f3 = torch.as_tensor(np.fft.rfft2(np.stack([initial_condition(500 + b, n3, amp=IC_AMP) for b in range(64)])),
                         dtype=torch.complex64, device=dev)
    tsb, _ = _timed(torch, flush, lambda: E.lawson_rk4(f3, 256 * 4.6 / 2048, 256, pd3s))
    # the precision target: Newton-GMRES with FP32 Jacobian products and FP64
    # residuals/Arnoldi/least squares, then FP64 refinement, from the reference's
    # 256^2 RPO2 (Re=50, 768 steps) perturbed by 1e-7
    from ecs_mhd_2d_b200 import drivers
    from ecs_mhd_2d_b200.utils import relative_error_RPO
    d = np.load(os.path.join(ROOT, "tests", "golden", "solution_Re50_RPO2.npz"))
    kw = dict(num_checkpoints=int(d["num_checkpoints"]), ministeps=int(d["ministeps"]),
              shift_reflect_ny=int(d["shift_reflect_ny"]), rot=bool(d["rot"]))
    pdr = E.make_param_dict(n3, float(d["nu"]), float(d["eta"]), b0=d["b0"], forcing="kolmogorov", **kw)
    u = E.dealias(torch.as_tensor(d["fields"] + 1e-7 * initial_condition(98, n3, amp=1.0), device=dev), pdr)
    x0 = {"fields": u, "T": float(d["T"]) * (1 + 1e-7), "sx": float(d["sx"])}
    r0 = float(relative_error_RPO(x0, E.objective_RPO(x0, pdr, "Lawson_RK4")))
    torch.cuda.synchronize()
    tn0 = time.perf_counter()
    _, hist = drivers.mixed_precision_newton(x0, pdr, "Lawson_RK4", iters=4, inner=32, refine=2)
    torch.cuda.synchronize()
    out["config3_newton_n256"] = {"start_rel_residual": r0, "final_rel_residual_fp64": hist[-1]["final_rel_err"],
                                  "per_step_rel_residual": [h.get("rel_err") for h in hist[:-1]],
                                  "jacobian": [h.get("jacobian") for h in hist[:-1]], "inner": 32,
                                  "seconds": time.perf_counter() - tn0,
                                  "base": "reference RPO2 (solutions/Re50/RPO2.npz), 768 Lawson-RK4 steps, +1e-7"}
    out["config3_mixed_n256"] = {"fp32_batch64_state_steps_per_s": 64 * 256 / tsb,
                                 "fp32_objective_steps_per_s": 2048 / t32, "fp64_objective_steps_per_s": 2048 / t64,
                                 "fp32_vs_fp64_objective_rel_err": err, "matvec_batch": Bt, "steps": 2048,
                                 "fp32_batch_matvecs_per_s": Bt / tj32, "fp64_batch_matvecs_per_s": Bt / tj64,
                                 "plain_fp64_b1_matvecs_per_s": 1.0 / tb1,
                                 "fp32_vs_fp64_tangent_rel_err": terr,
                                 "speedup_fp32_batch_vs_plain_fp64": (Bt / tj32) * tb1}
    return out


def plain_vs_batched(E, torch, dev, flush, prim, tan):
    """The 128^2 matvec workload as plain FP64 GMRES issues it, one tangent at a
    time at a fixed linearisation (linearisation excluded: amortised over the
    Krylov iterations), against the headline's batch (linearisation included)."""
    obj = E.Objective(param_dict(E), "Lawson_RK43")
    obj.linearize(prim, force=True, batch=1)
    t1 = {"fields": tan["fields"][:1].contiguous(), "T": tan["T"][:1], "sx": tan["sx"][:1]}
    tb1, _ = _timed(torch, flush, lambda: obj.jvp(prim, t1))
    tb, _ = _timed(torch, flush, lambda: obj.linearize_jvp(prim, tan)[1])
    B = tan["fields"].shape[0]
    return {"plain_fp64_b1_matvecs_per_s": 1.0 / tb1, "fp64_batch_matvecs_per_s": B / tb, "batch": B,
            "speedup_batch_vs_plain": (B / tb) * tb1}


def tdrk4_matvecs(E, torch, dev, flush, prim, tan):
    """Matvecs in TDRK4 mode (the reference Newton driver's default,
    jax_scripts/newton.py:70) on the same base point and tangents: 40 x 32 fixed
    steps over T=4.6, linearisation included, 64 tangents per batch."""
    pd = E.make_param_dict(N, 1 / RE, 1 / RE, forcing="kolmogorov+", num_checkpoints=40, ministeps=32,
                           shift_reflect_ny=0, rot=False)
    obj = E.Objective(pd, "TDRK4")
    t, o = _timed(torch, flush, lambda: obj.linearize_jvp(prim, tan)[1])
    B = tan["fields"].shape[0]
    return {"matvecs_per_s": B / t, "seconds": t, "steps": 1280, "batch": B,
            "finite": bool(torch.isfinite(o["fields"]).all())}


def dns_generation(E, torch, dev, flush):
    """DNS data generation in the reference script's configuration
    (jax_scripts/generate_turbulence.py: n=128 FP64, dt=1/256, Lawson-RK6,
    8192 transient steps, 256 snapshots of 64 steps, 256 x 256 recurrence):
    one trajectory (as the script runs it) and 64 independent trajectories,
    each timed over 1024 steps, and the recurrence matrix of 256 snapshots."""
    from ecs_mhd_2d_b200 import turbulence
    n, dt, S = 128, 1 / 256, 1024
    pd = E.make_param_dict(n, 1 / 40, 1 / 40, b0=(0.0, 0.3), forcing="kolmogorov")
    rng = np.random.default_rng(111111)
    f1 = torch.as_tensor(np.fft.rfft2(10.0 * rng.standard_normal((1, 2, n, n))), device=dev) * pd["mask"].to(dev)
    f1 = E.integrate(f1, dt * 512, 512, pd, "Lawson_RK6")              # leave the random initial data
    f64 = f1.repeat(64, 1, 1, 1) * (1 + 1e-3 * torch.arange(64, device=dev).view(64, 1, 1, 1))
    t1, _ = _timed(torch, flush, lambda: E.integrate(f1, dt * S, S, pd, "Lawson_RK6"))
    t64, _ = _timed(torch, flush, lambda: E.integrate(f64, dt * S, S, pd, "Lawson_RK6"))
    fs = E.integrate(f64, dt * 64, 64, pd, "Lawson_RK6").repeat(4, 1, 1, 1).contiguous()   # 256 snapshots
    tr, _ = _timed(torch, flush, lambda: turbulence.recurrence(fs, pd))
    script_steps = 8192 + 256 * 64
    return {"rk6_steps_per_s_b1": S / t1, "rk6_state_steps_per_s_b64": 64 * S / t64,
            "recurrence_256_ms": tr * 1e3, "script_steps": script_steps,
            "script_estimate_s": script_steps * t1 / S + tr}


def cpu_baseline_dns(steps=64):
    """The oracle's Lawson-RK6 (numpy) on the host for a few steps of the same
    128^2 FP64 DNS: steps per second of one trajectory."""
    import oracle as O
    n = 128
    opd = O.make_param_dict(n, 1 / 40, 1 / 40, b0=(0.0, 0.3), forcing="kolmogorov")
    f = np.fft.rfft2(10.0 * np.random.default_rng(111111).standard_normal((2, n, n))) * opd["mask"]
    v = lambda x: O.state_vel(x, opd, False)
    L = O.dissipation(opd)
    O.lawson_rk6(f, 1 / 256, 1, v, L, opd["mask"])
    t0 = time.perf_counter()
    O.lawson_rk6(f, steps / 256, steps, v, L, opd["mask"])
    t = time.perf_counter() - t0
    return {"value": steps / t, "unit": "steps/s", "cores": 1, "kind": "port",
            "sample": f"{steps} Lawson-RK6 steps of one 128^2 trajectory, {t:.2f} s, numpy oracle"}


def cpu_baseline(target_s=12.0, attempts_full=None):
    """The oracle (torch-CPU restatement, torch.func.jvp) on the host cores for a
    bounded sample: the first k attempts of the same adaptive JVP, scaled to one
    full matvec by the attempt count of the full solve."""
    import torch
    from torch.func import jvp
    import oracle as O
    torch.set_num_threads(os.cpu_count() or 1)
    u0, tv = host_inputs(0)

    def run(cap):
        ad = {"atol": ATOL, "checkpoints": 1, "max_steps_per_checkpoint": cap}
        pdt = O.make_param_dict(N, 1 / RE, 1 / RE, forcing="kolmogorov+", xp=O.TORCH, shift_reflect_ny=0,
                                rot=False, adaptive_dict=ad)
        prim = {"fields": torch.from_numpy(u0), "T": torch.tensor(T0, dtype=torch.float64),
                "sx": torch.tensor(SX0, dtype=torch.float64)}
        tan = {"fields": torch.from_numpy(tv[0, 1:-1].reshape(2, N, N)), "T": torch.tensor(tv[0, 0]),
               "sx": torch.tensor(tv[0, -1])}
        f = lambda d: O.objective_RPO(d, pdt, "Lawson_RK43", xp=O.TORCH)
        t0 = time.perf_counter()
        jvp(f, (prim,), (tan,))
        return time.perf_counter() - t0

    run(4)                                   # warm-up of the CPU FFT plans
    t_small = run(10)
    per = t_small / 10
    k = int(max(10, min(400, target_s / max(per, 1e-6))))
    t = run(k)
    per = t / k
    full = attempts_full or 1
    return {"value": 1.0 / (per * full), "unit": UNIT, "cores": torch.get_num_threads(), "kind": "port",
            "sample": f"first {k} attempts of one JVP (1 tangent) of the same workload, {t:.1f} s; "
                      f"scaled by {full} attempts per full matvec; restated oracle on CPU (torch.func.jvp), not JAX"}


REF_BUDGET_S = 150.0   # the reference arm starts no new timed step after this much timed CPU work


def oracle_matvec_fn():
    """One complete matvec of the workload as the reference computes it: jax.jvp
    of objective_RPO at the base point for one tangent (jax_scripts/lib/utils.py:108,
    called once per Arnoldi step by jax_scripts/newton.py:165), i.e. the adaptive
    primal solve and the tangent together.  Here torch.func.jvp of the oracle's
    torch form on the host cores.  Returns f(i, cap=None): the matvec of tangent
    i of the batch (cap: attempt cap override, for short warm-up runs)."""
    import torch
    from torch.func import jvp
    import oracle as O
    torch.set_num_threads(os.cpu_count() or 1)
    u0, tv = host_inputs(0)

    def f(i, cap=None):
        ad = {"atol": ATOL, "checkpoints": CAP[0] if cap is None else 1,
              "max_steps_per_checkpoint": CAP[1] if cap is None else cap}
        pdt = O.make_param_dict(N, 1 / RE, 1 / RE, forcing="kolmogorov+", xp=O.TORCH, shift_reflect_ny=0,
                                rot=False, adaptive_dict=ad)
        prim = {"fields": torch.from_numpy(u0), "T": torch.tensor(T0, dtype=torch.float64),
                "sx": torch.tensor(SX0, dtype=torch.float64)}
        t = tv[i % BATCH]
        tan = {"fields": torch.from_numpy(np.ascontiguousarray(t[1:-1].reshape(2, N, N))),
               "T": torch.tensor(t[0]), "sx": torch.tensor(t[-1])}
        jvp(lambda d: O.objective_RPO(d, pdt, "Lawson_RK43", xp=O.TORCH), (prim,), (tan,))
    return f


def run_reference(args, rank, budget_s=None):
    """The reference arm: the reference's CPU algorithm (the oracle; jax is not
    installable here) on this workload, one complete single-tangent matvec per
    step.  W warm-up steps are short (10-attempt) JVPs that build the FFT plans;
    then up to K complete matvecs are timed, stopping early once the timed work
    passes the budget (the line's steps / warmup are the counts actually run)."""
    if rank != 0:
        return
    budget_s = REF_BUDGET_S if budget_s is None else budget_s
    f = oracle_matvec_fn()
    for i in range(args.warmup):
        f(i, cap=10)
    times = []
    while len(times) < max(1, args.steps):
        t0 = time.perf_counter()
        f(len(times))
        times.append(time.perf_counter() - t0)
        if sum(times) + statistics.mean(times) > budget_s:
            break
    total = sum(times)
    value = len(times) / total
    import torch
    cores = torch.get_num_threads()
    sample = (f"{len(times)} complete matvecs (jax.jvp semantics: adaptive primal solve + 1 tangent, "
              f"torch.func.jvp of the oracle) of the workload, {total:.1f} s; restated oracle on CPU, not JAX")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": total / len(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded initial condition and tangents)", "config": workload_config(),
            "step": {"matvecs": 1, "what": "one jax.jvp of objective_RPO (primal solve + one tangent)",
                     "requested_steps": args.steps, "warmup_what": "10-attempt JVPs (FFT plans)",
                     "budget_s": budget_s},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serving_workload(requests=512, rate=40.0, seed=0):
    """Serving workload: a seeded Poisson stream of mixed requests {forward
    shooting, GMRES matvec, adjoint gradient} x n in {64,128,256} x horizons
    256-2048 steps x Re in {40,50}; n=256 runs FP32 stepping, the rest FP64, a
    quarter of the FP64 requests the adaptive Lawson_RK43 stepper.  Returns
    throughput, p50/p99 latency overall and per kind, and the batch sizes of
    the matvec sweeps."""
    import torch
    from ecs_mhd_2d_b200 import serving
    warm = serving.poisson_requests(9, rate=1000.0, seed=1000 + seed, horizons=(64,))
    serving.Server(slots=8, chunk_steps=32).run(warm)
    reqs = serving.poisson_requests(requests, rate=rate, seed=seed)
    srv = serving.Server(hbm_budget=96 << 30, slots=16, chunk_steps=32, workers_per_group=4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = srv.run(reqs)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    lat = np.array([r.latency for r in res])
    by = {}
    for k in ("forward", "matvec", "gradient"):
        lk = np.array([r.latency for r in res if r.kind == k])
        if lk.size:
            by[k] = {"count": int(lk.size), "p50_s": float(np.percentile(lk, 50)), "p99_s": float(np.percentile(lk, 99))}
    sweeps = {}
    for k in ("matvec", "gradient"):
        sw = [x for bt in srv.batchers.values() if bt.kind == k for x in bt.sweeps]
        sweeps[k] = {"sweeps": len(sw), "batch_mean": float(np.mean(sw)) if sw else None,
                     "batch_max": max(sw) if sw else None}
    return {"requests": len(res), "wall_s": wall, "requests_per_s": len(res) / wall,
            "arrival_rate_per_s": rate, "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "by_kind": by,
            "adaptive_requests": sum(r.mode == "Lawson_RK43" for r in reqs),
            "batched_sweeps": sweeps, "slots_per_pool": 16, "workers_per_group": 4}


def run_serving(args, rank, local, world):
    """`--workload serving`: the serving workload alone, one line; each rank
    serves its own stream (replicas); value = all requests / max time."""
    import torch
    import torch.distributed as dist
    from ecs_mhd_2d_b200 import build as _build
    _build.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    out = serving_workload(args.requests, args.rate, seed=rank)
    wall = max_over_ranks(out["wall_s"], world, "cuda")
    if rank == 0:
        line = {"metric": "serving throughput (mixed shooting requests)", "value": whole_job_rate(world, out["requests"], wall),
                "unit": "requests/s", "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": wall * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
                "data": "synthetic Poisson stream (seeded)",
                "config": {"workload": "serving_poisson_mixed", "requests": out["requests"],
                           "arrival_rate_per_s": args.rate, "n": [64, 128, 256], "horizons": [256, 512, 1024, 2048],
                           "Re": [40, 50]},
                "details": out}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_kernels(rank, local, B=64):
    """Profiling case: each hot kernel family once or a few times at n=128 FP64
    with a batch of 64 (the working sets of the batched passes are 30-60 MB,
    below the 126 MB L2, so DRAM counts of these launches are lower bounds):
    Lawson-RK4 stepping (k_col_rk4, k_row_rhs), the adaptive solve (k_col_rk43,
    k_row_err), linearisation + JVP batch (k_col_regen, k_row_phys, k_col_tan,
    k_row_tan), VJP batch (k_col_adj, k_row_adj), an Arnoldi step
    (k_arnoldi_mgs), a multi-candidate matvec sweep, and the batch-1 chains
    (k_tan_chain, k_rk4_chain).  Prints one JSON line with the seconds taken."""
    import torch
    import ecs_mhd_2d_b200 as E
    from ecs_mhd_2d_b200 import build as _build, linalg
    from ecs_mhd_2d_b200.synthetic import initial_condition
    _build.build()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    t0 = time.perf_counter()
    pd = E.make_param_dict(N, 1 / RE, 1 / RE, forcing="kolmogorov+", num_checkpoints=1, ministeps=8,
                           shift_reflect_ny=0, rot=False)
    f = torch.as_tensor(np.fft.rfft2(np.stack([initial_condition(b, N, amp=IC_AMP) for b in range(B)])), device=dev)
    E.lawson_rk4(f, 0.016, 8, pd)
    ad = {"atol": 1e-8, "checkpoints": 2, "max_steps_per_checkpoint": 16}
    pda = E.make_param_dict(N, 1 / RE, 1 / RE, forcing="kolmogorov+", shift_reflect_ny=0, rot=False, adaptive_dict=ad)
    u0, tv = host_inputs(rank)
    fields = torch.as_tensor(np.stack([initial_condition(b, N, amp=IC_AMP) for b in range(B)]), device=dev)
    E.objective_RPO({"fields": fields, "T": torch.full((B,), 0.05, dtype=torch.float64), "sx": 0.1}, pda, "Lawson_RK43")
    prim = {"fields": torch.as_tensor(u0, device=dev), "T": 0.05, "sx": SX0}
    tan = {"fields": torch.as_tensor(tv[:, 1:-1].reshape(BATCH, 2, N, N), device=dev).contiguous(),
           "T": torch.as_tensor(tv[:, 0]), "sx": torch.as_tensor(tv[:, -1])}
    obj = E.Objective(pda, "Lawson_RK43")
    obj.linearize_jvp(prim, tan)
    _, jacT = E.vjp(obj, prim)
    jacT(tan)
    x = torch.as_tensor(tv[0], device=dev)
    linalg.gmres(lambda v: v * 1.5 + 0.1 * torch.roll(v, 1), x, 8)
    pds = [E.make_param_dict(N, 1 / RE, 1 / RE, forcing="kolmogorov+", num_checkpoints=2, ministeps=8,
                             shift_reflect_ny=0, rot=False) for _ in range(16)]
    prims = [{"fields": fields[b], "T": 0.03, "sx": 0.1} for b in range(16)]
    tans = [{"fields": tan["fields"][b], "T": 0.1, "sx": 0.2} for b in range(16)]
    E.jvp_multi(prims, tans, pds)
    # batch-1 chains: the tangent pass list at the fixed linearisation (k_tan_chain)
    # and Lawson-RK4 stepping of one state (k_rk4_chain)
    obj.linearize(prim, force=True, batch=1)
    obj.jvp(prim, {"fields": tan["fields"][:1].contiguous(), "T": tan["T"][:1], "sx": tan["sx"][:1]})
    E.lawson_rk4(f[:1].contiguous(), 0.016, 8, pd)
    torch.cuda.synchronize()
    print(json.dumps({"workload": "kernels", "seconds": time.perf_counter() - t0}), flush=True)


def tangent_kernel_bytes(K, M, Bg, n=N, w=8):
    """Algorithmic bytes of one launch of the tangent row and column passes for a
    group of Bg tangents in the box layout (n=128 FP64: K=43, M=85): the row
    pass reads G (4 fields of K x n complex) and writes H (3 fields) per
    tangent and reads the shared primal fields (4 real n x n); the column pass
    reads H, writes G and reads/writes two box vectors of 2 K M complex per
    tangent, plus one shared record vector."""
    cb = 2 * w
    vec = 2 * K * M
    row = Bg * (4 + 3) * K * n * cb + n * 4 * n * w
    col = Bg * (3 * K * n * cb + 4 * K * n * cb + 2 * vec * cb) + vec * cb
    return row, col


# bytes of one tangent right-hand side of one tangent in the full-spectrum HBM
# model: 2 x B_rhs, B_rhs = 2 S + 4 Nr w with S = 4 Ns w (n=128 FP64: 1,056,768 B)
def tangent_rhs_model_bytes(n=N, w=8):
    ns, nr = n * (n // 2 + 1), n * n
    return 2 * (2 * 4 * ns * w + 4 * nr * w)


def kernel_roofline(E, torch, ctx, obj, prim, tan, flush, info):
    """Roofline row of the dominant tangent kernel, from one instrumented step."""
    import ctypes
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured (MEASURED_PEAKS.json hbm_gbs, copy)" if "hbm_gbs" in peaks else "fallback"
    flush.zero_()
    torch.cuda.synchronize()
    ctx.call("ecs_kernel_timing", 1, None, None, None, None, None)
    obj.linearize_jvp(prim, tan)
    torch.cuda.synchronize()
    rms, rn, cms, cn, bg = ctypes.c_double(), ctypes.c_int(), ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    ctx.call("ecs_kernel_timing", 0, ctypes.byref(rms), ctypes.byref(rn), ctypes.byref(cms), ctypes.byref(cn),
               ctypes.byref(bg))
    Bg = bg.value
    rb, cbytes = tangent_kernel_bytes(ctx.K, ctx.M, Bg)
    kern = {"k_row_tan": {"ms_per_launch": rms.value, "launches": rn.value, "bytes_per_launch": rb},
            "k_col_tan": {"ms_per_launch": cms.value, "launches": cn.value, "bytes_per_launch": cbytes}}
    for k in kern.values():
        k["GBps"] = k["bytes_per_launch"] / (k["ms_per_launch"] / 1e3) / 1e9 if k["ms_per_launch"] > 0 else None
        k["frac"] = k["GBps"] / hbm_peak if k["GBps"] else None
        k["total_ms"] = k["ms_per_launch"] * k["launches"]
    dom_name = max(kern, key=lambda k: kern[k]["total_ms"])
    dom = kern[dom_name]
    traffic, traffic_src = None, None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            t = json.load(open(tfile))[dom_name]
            traffic = t["fixed_bytes"] + t["bytes_per_tangent"] * Bg
            traffic_src = t["source"]
        except Exception:
            traffic = None
    pair_ms = rms.value + cms.value
    model = Bg * tangent_rhs_model_bytes()
    return {"bound": "hbm", "kernel": dom_name, "achieved": dom["GBps"], "peak": hbm_peak, "unit": "GB/s",
            "frac": dom["frac"], "traffic": traffic, "traffic_source": traffic_src, "peak_source": peak_src,
            "algorithmic_bytes_per_launch": dom["bytes_per_launch"], "ms_per_launch": dom["ms_per_launch"],
            "how": "CUDA events around tangent group 0's launches in one instrumented step "
                   f"(group of {Bg} tangents; the other groups run beside it); bytes: box layout",
            "group_batch": Bg, "kernels": kern,
            "tangent_rhs_model": {"bytes_per_pair": model, "pair_ms": pair_ms,
                                  "GBps": model / (pair_ms / 1e3) / 1e9 if pair_ms > 0 else None,
                                  "frac": (model / (pair_ms / 1e3) / 1e9) / hbm_peak if pair_ms > 0 else None,
                                  "what": "one row + one column launch = one tangent RHS per tangent; "
                                          "bytes = group x 2 x B_rhs of the full-spectrum HBM model"}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="skip the config 0/2/3 side measurements")
    ap.add_argument("--workload", default="matvec", choices=["matvec", "serving", "kernels"],
                    help="matvec: the headline 128^2 matvec batch; serving: 512 mixed Poisson requests; "
                         "kernels: one short pass over every hot kernel family (profiling case)")
    ap.add_argument("--requests", type=int, default=512)
    ap.add_argument("--rate", type=float, default=40.0, help="serving: Poisson arrival rate (requests/s)")
    ap.add_argument("--T", type=float, default=None, help="profiling only: shorter horizon (small ncu case)")
    ap.add_argument("--cap", type=int, nargs=2, default=None, help="profiling only: checkpoints max_steps")
    args = ap.parse_args()
    global T0, CAP
    if args.T is not None:
        T0 = args.T
    if args.cap is not None:
        CAP = tuple(args.cap)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "serving":
        run_serving(args, rank, local, world)
        return
    if args.workload == "kernels":
        run_kernels(rank, local)
        return

    import torch
    import torch.distributed as dist
    import ecs_mhd_2d_b200 as E
    from ecs_mhd_2d_b200 import build as _build, context as C
    _build.build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    pd = param_dict(E)
    u0h, tvh = host_inputs(rank)
    dev = torch.device("cuda", local)
    prim = {"fields": torch.as_tensor(u0h, device=dev), "T": T0, "sx": SX0}
    tan = {"fields": torch.as_tensor(tvh[:, 1:-1].reshape(BATCH, 2, N, N), device=dev).contiguous(),
           "T": torch.as_tensor(tvh[:, 0]), "sx": torch.as_tensor(tvh[:, -1])}
    obj = E.Objective(pd, "Lawson_RK43")

    def step():   # primal solve with record overlapped with the 64-tangent sweep (jax.jvp semantics)
        return obj.linearize_jvp(prim, tan)[1]

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    info = dict(obj.last_info)
    ctx = obj._ctx
    lib = ctx.lib
    n_launch0 = lib.ecs_launch_count(ctx.handle)

    def barrier():
        if world > 1:
            dist.barrier()

    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            step()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    launches = lib.ecs_launch_count(ctx.handle) - n_launch0
    t_total = max_over_ranks(sum(times), world, dev)
    ms_per_step = t_total / args.steps
    value = whole_job_rate(world, BATCH * args.steps, t_total / 1e3)

    # end to end through the public API from pinned host buffers
    u0_pin = torch.as_tensor(u0h).pin_memory()
    tf_pin = torch.as_tensor(tvh[:, 1:-1].reshape(BATCH, 2, N, N)).contiguous().pin_memory()
    tT_pin, tsx_pin = torch.as_tensor(tvh[:, 0]).pin_memory(), torch.as_tensor(tvh[:, -1]).pin_memory()
    out_pin = torch.empty((BATCH, 2, N, N), dtype=torch.float64).pin_memory()
    oT_pin = torch.empty(BATCH, dtype=torch.float64).pin_memory()
    h2d = u0_pin.numel() * 8 + tf_pin.numel() * 8 + 2 * BATCH * 8 + 16
    d2h = out_pin.numel() * 8 + 2 * BATCH * 8
    e2e_times = []
    for it in range(args.warmup + args.steps):   # the same untimed warm-up as the device-resident loop
        flush.zero_()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        p = {"fields": u0_pin.to(dev, non_blocking=True), "T": T0, "sx": SX0}
        tg = {"fields": tf_pin.to(dev, non_blocking=True), "T": tT_pin.to(dev, non_blocking=True),
              "sx": tsx_pin.to(dev, non_blocking=True)}
        o = obj.linearize_jvp(p, tg)[1]
        out_pin.copy_(o["fields"], non_blocking=True)
        oT_pin.copy_(o["T"], non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        if it >= args.warmup:
            e2e_times.append(e0.elapsed_time(e1))
    te = max_over_ranks(sum(e2e_times), world, dev)
    e2e_value = whole_job_rate(world, BATCH * args.steps, te / 1e3)

    # phase split of one step (untimed pass, CUDA events): primal linearisation vs tangent sweep
    def _ev_ms(fn):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b)
    phase_ms = {"linearize": _ev_ms(lambda: obj.linearize(prim, force=True, batch=BATCH)),
                "jvp": _ev_ms(lambda: obj.jvp(prim, tan))}

    # roofline of the dominant kernel in the step's own launch shape: one more
    # (untimed) step with CUDA events around tangent group 0's row-pass and
    # column-pass launches of every accepted attempt, on that group's stream
    # (the other groups run beside it, as in the timed steps)
    roofline = kernel_roofline(E, torch, ctx, obj, prim, tan, flush, info)

    # secondary: Lawson-RK4 state-steps/s at 128^2 FP64 (batch 64 and a single state)
    def rk4_rate(B, S=64):
        from ecs_mhd_2d_b200.synthetic import initial_condition
        pd4 = E.make_param_dict(N, 1 / RE, 1 / RE, forcing="kolmogorov+")
        f = torch.as_tensor(np.fft.rfft2(np.stack([initial_condition(1000 + b, N, amp=IC_AMP) for b in range(B)])),
                            device=dev)
        E.lawson_rk4(f, 0.002 * S, S, pd4)
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        E.lawson_rk4(f, 0.002 * S, S, pd4)
        e1.record()
        torch.cuda.synchronize()
        return B * S / (e0.elapsed_time(e1) / 1e3)
    rk4_b64, rk4_b1 = rk4_rate(64), rk4_rate(1)
    secondary = secondary_workloads(E, torch, dev, flush) if not args.no_secondary else {}
    if not args.no_secondary:
        secondary["config1_plain_vs_batched"] = plain_vs_batched(E, torch, dev, flush, prim, tan)
        secondary["tdrk4_matvec_n128_f64"] = tdrk4_matvecs(E, torch, dev, flush, prim, tan)
        secondary["dns_generation_n128_f64"] = dns_generation(E, torch, dev, flush)
        secondary["serving_poisson_512"] = serving_workload(args.requests, args.rate, seed=rank)

    if rank == 0:
        clocks = clk.summary()
        cb = None
        if not args.no_cpu_baseline:
            try:
                cb = cpu_baseline(attempts_full=info.get("accepted", 0) + info.get("rejected", 0))
            except Exception as ex:  # the oracle is test infrastructure; report why it is missing
                cb = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}
            if "dns_generation_n128_f64" in secondary:
                try:
                    secondary["dns_generation_n128_f64"]["cpu_baseline"] = cpu_baseline_dns()
                except Exception as ex:
                    secondary["dns_generation_n128_f64"]["cpu_baseline"] = {"value": None, "sample": f"failed: {ex}"}
        details = {"adaptive_info": info, "rk_attempts_per_matvec": info.get("accepted", 0) + info.get("rejected", 0),
                   "tangent_rk_steps_per_s": value * info.get("accepted", 0),
                   "lawson_rk4_state_steps_per_s": {"batch64": rk4_b64, "batch1": rk4_b1},
                   "phase_ms": phase_ms, "secondary": secondary}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded initial condition and tangents)",
                "config": workload_config(),
                "step": {"matvecs": BATCH, "what": "one jax.jvp of objective_RPO with a batch of 64 tangents "
                                                   "(primal solve + 64 tangents, overlapped)"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": int(launches), "clocks": clocks, "roofline": roofline, "cpu_baseline": cb,
                "details": details}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
