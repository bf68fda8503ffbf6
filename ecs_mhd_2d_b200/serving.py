"""Continuous-batching request server for shooting requests.

Request kinds (one RPO candidate each): "forward" (objective_RPO residual and
loss_RPO), "matvec" (one JVP of objective_RPO, the Newton-GMRES matvec) and
"gradient" (loss_RPO and its gradient by the adjoint kernels).  Requests carry
their own grid n, horizon (steps), Reynolds number, T, sx and state.

* Forward requests join a slot pool of their (n, dtype, physics) group
  (ecs_pool_*): every slot has its own step size and budget, finished slots are
  skipped, and new requests are admitted at step boundaries while the other
  slots keep running — continuous batching, not a queue.
* Matvec and gradient requests in Lawson_RK4 mode go to their group's
  batchers: whatever has queued while a batcher's previous sweep ran (up to its
  batch size) becomes the next sweep over all those candidates, each with its
  own state, T, sx and horizon — one forward-mode pass for matvecs
  (ecs_jvp_multi), one forward pass and one adjoint pass for gradients
  (ecs_loss_grad_multi).
* Requests in adaptive Lawson_RK43 mode run on worker threads, each with a
  private context and CUDA stream, so several linearisations proceed
  concurrently (adaptive candidates do not step in lockstep).
* Admission is by HBM footprint: a request is admitted only while the
  estimated device memory of all live contexts and records stays within the
  budget; otherwise it waits.

Work of different groups runs on different streams and overlaps on the GPU.
"""

from __future__ import annotations

import ctypes
import dataclasses
import queue
import threading
import time

import numpy as np
import torch

from . import _lib
from . import context as C
from .autodiff import Objective, jvp_multi, loss_and_grad, loss_grad_multi
from .loss_functions import objective_RPO, shoot_cfg
from .mhd import make_param_dict


@dataclasses.dataclass
class Request:
    rid: int
    kind: str                  # "forward" | "matvec" | "gradient"
    n: int
    steps: int                 # Lawson-RK4 steps over [0, T]
    Re: float
    T: float
    sx: float
    fields: np.ndarray         # [2, n, n] float64 (host)
    tangent: np.ndarray = None  # matvec: flat [T, fields, sx] (host)
    arrival: float = 0.0       # seconds after the start of the run
    dtype: torch.dtype = torch.float64
    mode: str = "Lawson_RK4"   # or "Lawson_RK43" (adaptive, tolerance atol; T as for the fixed-step horizon)
    atol: float = 1e-6


@dataclasses.dataclass
class Result:
    rid: int
    kind: str
    out: dict
    t_arrival: float
    t_admit: float
    t_done: float

    @property
    def latency(self):
        return self.t_done - self.t_arrival


def _nc_ms(steps):
    ms = 32 if steps % 32 == 0 else steps
    return steps // ms, ms


def _ckpt(req):
    """Matvecs keep the full record (their primal solve overlaps the tangent
    sweep); gradients keep one state per ministeps segment."""
    return 0 if req.kind == "matvec" else _nc_ms(req.steps)[1]


ADAPTIVE_CAP = (64, 64)   # checkpoints x max_steps_per_checkpoint of adaptive requests


def _param_dict(req, dtype):
    nc, ms = _nc_ms(req.steps)
    ad = {"atol": req.atol, "checkpoints": ADAPTIVE_CAP[0], "max_steps_per_checkpoint": ADAPTIVE_CAP[1]}
    return make_param_dict(req.n, 1.0 / req.Re, 1.0 / req.Re, forcing="kolmogorov+", data_type=dtype,
                           num_checkpoints=nc, ministeps=ms, shift_reflect_ny=0, rot=False, ckpt_every=_ckpt(req),
                           adaptive_dict=ad)


def context_bytes(n, dtype, batch):
    """Device bytes of a context's workspace (ecs_ctx_create, ctx_init)."""
    K, M = (n - 1) // 3 + 1, 2 * ((n - 1) // 3) + 1
    rb = 8 if dtype == torch.float64 else 4
    cb = 2 * rb
    box = batch * 2 * K * M
    # F, A1, K2, OUT, V; Etab; G [B][4][K][n] and H [B][4][K][n]; three real field buffers; RK4(3) slots
    return (5 * box * cb + box * rb + 2 * batch * 4 * K * n * cb + 3 * batch * 2 * n * n * rb
            + 10 * box * cb + (64 << 20))


def record_bytes(n, dtype, steps, ckpt, mode="Lawson_RK4"):
    K, M = (n - 1) // 3 + 1, 2 * ((n - 1) // 3) + 1
    cb = 16 if dtype == torch.float64 else 8
    vec = 2 * K * M * cb
    regen = 384 << 20
    if mode == "Lawson_RK43":   # 11 record vectors per attempt up to the attempt cap
        return ADAPTIVE_CAP[0] * ADAPTIVE_CAP[1] * 11 * vec + regen
    seg = ckpt if ckpt else steps
    return seg * 8 * vec + (steps // max(seg, 1) + 1) * vec + regen


def grad_multi_bytes(n, dtype, batch, max_steps=2048, seg=32):
    """Device bytes of ecs_loss_grad_multi's buffers beyond multi_bytes:
    segment start states, one segment's record and stage fields, residuals."""
    K, M = (n - 1) // 3 + 1, 2 * ((n - 1) // 3) + 1
    rb = 8 if dtype == torch.float64 else 4
    vec = 2 * K * M * 2 * rb
    return batch * ((max_steps // seg) * vec + seg * 8 * vec + seg * 4 * n * 4 * n * rb + 4 * n * n * rb)


def multi_bytes(n, dtype, batch):
    """Device bytes of ecs_jvp_multi's buffers beyond the context workspace:
    tangent G/H, one stage's physical fields, one step's record, phase fields,
    tangent slots."""
    K, M = (n - 1) // 3 + 1, 2 * ((n - 1) // 3) + 1
    rb = 8 if dtype == torch.float64 else 4
    cb = 2 * rb
    return batch * (7 * K * n * cb + 4 * n * n * rb + 8 * 2 * K * M * cb + 4 * n * n * rb + 3 * 2 * K * M * cb)


class ForwardPool:
    """Slot pool of one (n, dtype, Re) group."""

    def __init__(self, n, dtype, Re, slots):
        self.n, self.dtype, self.Re, self.slots = n, dtype, Re, slots
        self.pd = make_param_dict(n, 1.0 / Re, 1.0 / Re, forcing="kolmogorov+", data_type=dtype)
        fk = C._forcing_key(self.pd["forcing"])
        self.ctx = C.Context(n, dtype, 1.0 / Re, 1.0 / Re, self.pd["b0"], fk[1], max_batch=slots)
        # high priority: the pool's small step launches run ahead of the batchers'
        # and workers' large sweeps instead of queueing behind them (the scheduler
        # waits for every pool's chunk before it admits and retires again)
        self.stream = torch.cuda.Stream(priority=-1)
        self.req = [None] * slots
        self.t_admit = [0.0] * slots
        self.bytes = context_bytes(n, dtype, slots)
        with torch.cuda.stream(self.stream):
            self.ctx.call("ecs_pool_reset", C.stream_ptr())

    def free_slot(self):
        for i, r in enumerate(self.req):
            if r is None:
                return i
        return -1

    def admit(self, req, now):
        slot = self.free_slot()
        nc, ms = _nc_ms(req.steps)
        pd = dict(self.pd, num_checkpoints=nc, ministeps=ms, shift_reflect_ny=0, rot=False)
        cfg = shoot_cfg(pd, "Lawson_RK4")
        with torch.cuda.stream(self.stream):
            f = torch.as_tensor(req.fields, dtype=self.dtype).to("cuda", non_blocking=True).contiguous()
            self.ctx.call("ecs_pool_admit", slot, cfg, C.ptr(f), float(req.T), float(req.sx), C.stream_ptr())
            self._keep = f
        self.req[slot] = req
        self.t_admit[slot] = now

    def active(self):
        return any(r is not None for r in self.req)

    def advance(self, nsteps):
        with torch.cuda.stream(self.stream):
            self.ctx.call("ecs_pool_advance", int(nsteps), C.stream_ptr())

    def harvest(self, now_fn):
        done = (ctypes.c_int * self.slots)()
        with torch.cuda.stream(self.stream):
            self.ctx.call("ecs_pool_poll", done, None, C.stream_ptr())
        out = []
        for i in range(self.slots):
            if self.req[i] is not None and done[i]:
                with torch.cuda.stream(self.stream):
                    res = torch.empty((2, self.n, self.n), dtype=self.dtype, device="cuda")
                    loss = torch.empty(1, dtype=torch.float64, device="cuda")
                    self.ctx.call("ecs_pool_retire", i, C.ptr(res), C.ptr(loss), C.stream_ptr())
                    self.stream.synchronize()
                r = self.req[i]
                out.append(Result(r.rid, r.kind, {"fields": res, "loss": float(loss[0])}, r.arrival,
                                  self.t_admit[i], now_fn()))
                self.req[i] = None
        return out


class Worker(threading.Thread):
    """Matvec / gradient requests of one (n, dtype, Re) group, one at a time,
    on a private context and stream."""

    def __init__(self, n, dtype, Re, results, now_fn):
        super().__init__(daemon=True)
        self.n, self.dtype, self.Re = n, dtype, Re
        self.inbox = queue.Queue()
        self.results, self.now_fn = results, now_fn
        self.busy = False
        self.req_bytes = 0
        self.bytes = context_bytes(n, dtype, 1)
        self.ctx = None
        self.stream = None
        self.error = None

    def run(self):
        torch.cuda.set_device(0)
        self.stream = torch.cuda.Stream()
        pd0 = make_param_dict(self.n, 1.0 / self.Re, 1.0 / self.Re, forcing="kolmogorov+", data_type=self.dtype)
        fk = C._forcing_key(pd0["forcing"])
        self.ctx = C.Context(self.n, self.dtype, 1.0 / self.Re, 1.0 / self.Re, pd0["b0"], fk[1], max_batch=1)
        while True:
            item = self.inbox.get()
            if item is None:
                break
            req, t_admit = item
            try:
                out = run_adjoint_request(req, self.ctx, self.stream)
                self.results.put(Result(req.rid, req.kind, out, req.arrival, t_admit, self.now_fn()))
            except Exception as ex:   # surfaced by Server.run
                self.error = ex
                self.results.put(None)
            self.busy = False
        self.ctx.close()   # in this thread, before the interpreter's shutdown


class Batcher(threading.Thread):
    """Lawson_RK4 requests of one kind ("matvec" or "gradient") and one (n,
    dtype, Re) group: each sweep takes every request queued so far (up to
    `batch`) and runs them as one ecs_jvp_multi or ecs_loss_grad_multi call on a
    private context and stream, so requests that arrive during a sweep join the
    next one."""

    def __init__(self, kind, n, dtype, Re, results, now_fn, batch=16):
        super().__init__(daemon=True)
        self.kind, self.n, self.dtype, self.Re, self.batch = kind, n, dtype, Re, batch
        self.inbox = queue.Queue()
        self.results, self.now_fn = results, now_fn
        self.queued = 0                  # requests handed over and not yet finished
        self.lock = threading.Lock()     # guards `queued` (the scheduler adds, this thread subtracts)
        self.bytes = context_bytes(n, dtype, batch) + multi_bytes(n, dtype, batch)
        if kind == "gradient":
            self.bytes += grad_multi_bytes(n, dtype, batch)
        self.error = None
        self.sweeps = []   # batch size of every sweep run

    def run(self):
        torch.cuda.set_device(0)
        stream = torch.cuda.Stream()
        pd0 = make_param_dict(self.n, 1.0 / self.Re, 1.0 / self.Re, forcing="kolmogorov+", data_type=self.dtype)
        fk = C._forcing_key(pd0["forcing"])
        ctx = C.Context(self.n, self.dtype, 1.0 / self.Re, 1.0 / self.Re, pd0["b0"], fk[1], max_batch=self.batch)
        while True:
            item = self.inbox.get()
            if item is None:
                break
            items = [item]
            while len(items) < self.batch:
                try:
                    nxt = self.inbox.get_nowait()
                except queue.Empty:
                    break
                if nxt is None:
                    self.inbox.put(None)
                    break
                items.append(nxt)
            try:
                run = run_matvec_batch if self.kind == "matvec" else run_gradient_batch
                outs = run([r for r, _ in items], ctx, stream)
                self.sweeps.append(len(items))
                t = self.now_fn()
                for (req, t_admit), out in zip(items, outs):
                    self.results.put(Result(req.rid, req.kind, out, req.arrival, t_admit, t))
            except Exception as ex:   # surfaced by Server.run
                self.error = ex
                self.results.put(None)
            with self.lock:
                self.queued -= len(items)
        ctx.close()   # in this thread, before the interpreter's shutdown


def run_matvec_batch(reqs, ctx, stream):
    """Lawson_RK4 matvec requests of one group in one ecs_jvp_multi sweep."""
    with torch.cuda.stream(stream):
        prims, tans, pds = [], [], []
        for req in reqs:
            n = req.n
            prims.append({"fields": torch.as_tensor(req.fields, dtype=req.dtype).to("cuda").contiguous(),
                          "T": req.T, "sx": req.sx})
            tv = req.tangent
            tans.append({"fields": torch.as_tensor(tv[1:-1].reshape(2, n, n), dtype=req.dtype).to("cuda").contiguous(),
                         "T": float(tv[0]), "sx": float(tv[-1])})
            pds.append(_param_dict(req, req.dtype))
        _, jv = jvp_multi(prims, tans, pds, "Lawson_RK4", ctx=ctx)
        outs = [{"fields": j["fields"].clone(), "T": float(j["T"]), "sx": float(j["sx"])} for j in jv]
        stream.synchronize()
    return outs


def run_gradient_batch(reqs, ctx, stream):
    """Lawson_RK4 gradient requests of one group in one ecs_loss_grad_multi sweep."""
    with torch.cuda.stream(stream):
        xs = [{"fields": torch.as_tensor(r.fields, dtype=r.dtype).to("cuda").contiguous(), "T": r.T, "sx": r.sx}
              for r in reqs]
        res = loss_grad_multi(xs, [_param_dict(r, r.dtype) for r in reqs], "Lawson_RK4", ctx=ctx)
        outs = [{"loss": float(l), "fields": g["fields"].clone(), "T": float(g["T"]), "sx": float(g["sx"])}
                for l, g in res]
        stream.synchronize()
    return outs


def run_adjoint_request(req, ctx, stream):
    """One request on a single-candidate context `ctx` and `stream`: a matvec
    (JVP), a gradient (loss and its gradient by the adjoint), or, in adaptive
    mode, a forward shooting."""
    pd = _param_dict(req, req.dtype)
    with torch.cuda.stream(stream):
        x = {"fields": torch.as_tensor(req.fields, dtype=req.dtype).to("cuda").contiguous(), "T": req.T, "sx": req.sx}
        if req.kind == "forward":   # loss_RPO = mean(irfft2(f - f0)^2) of the same residual
            res = objective_RPO(x, pd, req.mode, ctx=ctx)["fields"]
            loss = torch.sum(res.double() ** 2) / (2 * req.n * req.n)
            out = {"fields": res.clone(), "loss": float(loss)}
        elif req.kind == "matvec":
            obj = Objective(pd, req.mode, ctx=ctx)
            n = req.n
            tv = req.tangent
            tan = {"fields": torch.as_tensor(tv[1:-1].reshape(2, n, n), dtype=req.dtype).to("cuda").contiguous(),
                   "T": float(tv[0]), "sx": float(tv[-1])}
            _, o = obj.linearize_jvp(x, tan)
            out = {"fields": o["fields"].clone(), "T": float(o["T"]), "sx": float(o["sx"])}
        else:
            (loss, info), g = loss_and_grad(x, pd, req.mode, ctx=ctx)
            out = {"loss": float(loss), "fields": g["fields"].clone(), "T": float(g["T"]), "sx": float(g["sx"])}
        stream.synchronize()
    return out


class Server:
    def __init__(self, hbm_budget=64 << 30, slots=16, chunk_steps=32, workers_per_group=4):
        self.budget, self.slots, self.chunk = hbm_budget, slots, chunk_steps
        self.workers_per_group = workers_per_group
        self.pools, self.workers, self.batchers = {}, {}, {}
        self.results = queue.Queue()

    def _used(self):
        return (sum(p.bytes for p in self.pools.values()) + sum(b.bytes for b in self.batchers.values())
                + sum(w.bytes + w.req_bytes for ws in self.workers.values() for w in ws))

    def run(self, requests, time_scale=1.0):
        """Serve `requests` (arrival times in seconds); returns results in rid order."""
        t0 = time.perf_counter()
        now = lambda: (time.perf_counter() - t0) / time_scale
        self._now = now
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting, results = [], {}
        total = len(pending)
        while len(results) < total:
            t = now()
            while pending and pending[0].arrival <= t:
                waiting.append(pending.pop(0))
            still = []
            for r in waiting:
                if not self._admit(r, t):
                    still.append(r)
            waiting = still
            for p in self.pools.values():
                if p.active():
                    p.advance(self.chunk)
            for p in self.pools.values():
                if p.active():
                    for res in p.harvest(now):
                        results[res.rid] = res
            while True:
                try:
                    res = self.results.get_nowait()
                except queue.Empty:
                    break
                if res is None:
                    raise RuntimeError([w.error for ws in self.workers.values() for w in ws if w.error]
                                       + [b.error for b in self.batchers.values() if b.error])
                results[res.rid] = res
            if not any(p.active() for p in self.pools.values()) and len(results) < total:
                time.sleep(0.0005)
        self.close()
        return [results[k] for k in sorted(results)]

    def close(self):
        """Stop the worker and batcher threads (each releases its context) and
        release the pools' contexts, so that nothing is left to tear down at
        interpreter exit.  The stopped batchers stay in `batchers` (their sweep
        sizes); a later run starts new threads and pools."""
        threads = [w for ws in self.workers.values() for w in ws] + list(self.batchers.values())
        for t in threads:
            if t.is_alive():
                t.inbox.put(None)
        for t in threads:
            t.join(timeout=120)
        for p in self.pools.values():
            p.ctx.close()
        self.workers, self.pools = {}, {}

    def _admit(self, r, t):
        key = (r.n, r.dtype, r.Re)
        if r.kind in ("matvec", "gradient") and r.mode == "Lawson_RK4":
            bkey = (r.kind,) + key
            bt = self.batchers.get(bkey)
            if bt is None or not bt.is_alive():   # (a batcher of an earlier run has stopped)
                need = context_bytes(r.n, r.dtype, self.slots) + multi_bytes(r.n, r.dtype, self.slots)
                if r.kind == "gradient":
                    need += grad_multi_bytes(r.n, r.dtype, self.slots)
                if self._used() + need > self.budget:
                    return False
                bt = self.batchers[bkey] = Batcher(r.kind, r.n, r.dtype, r.Re, self.results, self._now,
                                                   batch=self.slots)
                bt.start()
            with bt.lock:
                if bt.queued >= 2 * bt.batch:   # bounded backlog: the rest waits for admission
                    return False
                bt.queued += 1
            bt.inbox.put((r, t))
            return True
        if r.kind == "forward" and r.mode == "Lawson_RK4":
            pool = self.pools.get(key)
            if pool is None:
                need = context_bytes(r.n, r.dtype, self.slots)
                if self._used() + need > self.budget:
                    return False
                pool = self.pools[key] = ForwardPool(r.n, r.dtype, r.Re, self.slots)
            if pool.free_slot() < 0:
                return False
            pool.admit(r, t)
            return True
        ws = self.workers.setdefault(key, [])
        idle = [w for w in ws if not w.busy]
        need = record_bytes(r.n, r.dtype, r.steps, _ckpt(r), r.mode)
        if not idle:
            if len(ws) >= self.workers_per_group:
                return False
            if self._used() + context_bytes(r.n, r.dtype, 1) + need > self.budget:
                return False
            w = Worker(r.n, r.dtype, r.Re, self.results, self._now)
            w.start()
            ws.append(w)
            idle = [w]
        w = idle[0]
        if self._used() + need > self.budget:
            return False
        w.busy = True
        w.req_bytes = need
        w.inbox.put((r, t))
        return True


def poisson_requests(count, rate, seed=0, ns=(64, 128, 256), horizons=(256, 512, 1024, 2048), Res=(40.0, 50.0),
                     kinds=("forward", "matvec", "gradient"), fp32_for_256=True, adaptive_fraction=0.25,
                     adaptive_atol=1e-6):
    """Seeded Poisson stream of mixed requests (the serving workload).  A
    fraction of the FP64 requests (n < 256) runs the adaptive Lawson_RK43
    stepper with tolerance `adaptive_atol`; the rest, and every FP32 request,
    Lawson_RK4."""
    from .synthetic import initial_condition, unit_tangents
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        n = int(rng.choice(ns))
        steps = int(rng.choice(horizons))
        kind = str(rng.choice(kinds))
        dt = 0.005 * 64 / n
        req = Request(rid=i, kind=kind, n=n, steps=steps, Re=float(rng.choice(Res)), T=steps * dt,
                      sx=float(rng.uniform(-0.5, 0.5)), fields=initial_condition(int(rng.integers(1 << 30)), n, amp=2.0),
                      arrival=t, dtype=torch.float32 if (fp32_for_256 and n == 256) else torch.float64)
        if kind == "matvec":
            req.tangent = unit_tangents(int(rng.integers(1 << 30)), n, 1)[0]
        if rng.uniform() < adaptive_fraction and req.dtype == torch.float64:
            req.mode, req.atol = "Lawson_RK43", adaptive_atol
        out.append(req)
    return out
