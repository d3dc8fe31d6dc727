"""The multi-GPU form of bench.py is N independent replicas (the path does not shard across
devices in this build): each rank times its own step, the job's time is the maximum over
ranks and the job's rate counts every rank's work.  These are checked with two gloo ranks on
the CPU (127.0.0.1 rendezvous), as are the barrier and the reference arm's rank-0-only rule."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        my_ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
        bench.barrier(world)
        ms = bench.max_over_ranks(my_ms, world)
        rate = bench.job_tflops(world, 2.0e12, ms)
        buf = io.StringIO()
        with redirect_stdout(buf):
            args = type("A", (), {"gpus": world, "steps": 1, "warmup": 0, "size": 256})()
            if rank != 0:
                bench.reference_arm(args)  # non-zero ranks return without work or output
        bench.barrier(world)
        out.put((rank, ms, rate, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate, printed in results:
        assert ms == 15.0  # every rank agrees on the slowest replica's time
        assert rate == pytest.approx(2 * 2.0e12 / 15e-3 / 1e12)
        assert printed == ""
