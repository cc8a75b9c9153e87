"""Multi-rank protocol of the benchmark, on CPU with world-size-2 gloo
process groups: every rank contracts its own replica, the job's time is the
slowest rank's (one MAX all-reduce of a scalar, then a barrier), the job value
counts every rank's work, and the reference arm runs on rank 0 only while the
other ranks leave without work."""
import io
import os
import sys
import contextlib

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r "took" 10*(r+1) ms for its steps
        t = bench.max_over_ranks(dist, torch, 10.0 * (rank + 1), torch.device("cpu"))
        single = bench.max_over_ranks(None, torch, 3.0, torch.device("cpu"))
        value = bench.job_value(world, 5, t)
        # the reference arm: only rank 0 prints
        out = io.StringIO()
        with contextlib.redirect_stdout(out):
            args = bench.parse(["--impl", "reference", "--gpus", str(world), "--steps", "1", "--warmup", "0"])
            if rank != 0:
                bench.run_reference(args)
        dist.barrier()
        q.put((rank, t, single, value, out.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_and_value():
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    import bench
    port = 29500 + (os.getpid() % 1000)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, single, value, out in res:
        assert t == 20.0                      # the slowest rank's time on every rank
        assert single == 3.0
        assert value == pytest.approx(2 * bench.FLOPS_LADDER * 5 / 0.020 / 1e9)
        if rank != 0:
            assert out == ""                  # non-zero ranks of the reference arm print nothing
