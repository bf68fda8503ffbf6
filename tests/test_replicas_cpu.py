"""The multi-GPU form of the benchmark is N independent replicas (one process
per GPU, no data-path collective).  Its host-side rank logic runs here as two
gloo ranks on the CPU: the step time is the maximum over ranks, the value is
the whole job's units over that time, every rank works on its own seeded
inputs, and only rank 0 of the reference arm does work and prints."""
import contextlib
import io
import os
import socket
import sys

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        local_ms = [120.0, 150.0][rank]                  # per-rank timed region
        t_max = bench.max_over_ranks(local_ms, world, "cpu")
        value = bench.whole_job_rate(world, bench.BATCH * 3, t_max / 1e3)
        u0, tv = bench.host_inputs(rank)
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            if rank != 0:
                bench.run_reference(None, rank)           # non-zero ranks exit without work
        dist.barrier()
        out.put((rank, t_max, value, float(np.abs(u0).sum()), float(np.abs(tv).sum()), buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_replica_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, v0, a0, b0, o0), (r1, t1, v1, a1, b1, o1) = res
    sys.path.insert(0, ROOT)
    import bench
    assert t0 == t1 == 150.0                              # max over ranks, the same on every rank
    assert v0 == v1 == world * bench.BATCH * 3 / 0.150    # whole-job units / slowest rank
    assert a0 != a1 and b0 != b1                          # independent replica inputs
    assert o1 == ""                                       # only rank 0 of the reference arm prints
