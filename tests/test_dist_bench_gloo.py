"""The multi-GPU arm of the benchmark (dgt.dist.summa_benchmark, what `bench.py --gpus N`
runs for N > 1) as gloo ranks on the CPU: both forms of the physical SUMMA step loop --
collective (DistSumma, panel broadcasts) and fused (PeerSumma, peers' panels read in place)
-- run on the reference's most-square grid with host doubles for the rank-local
operations, the IPC buffers (process-shared memory) and the per-rank SUMMA kernel (the
segments dgt_summa_schedule gives).  Checked: the grid, positive times for every form and
the compute reference, and the two forms' results agreeing within 1e-13 (relative
Frobenius) after the same number of multiplies."""
import os
import sys

import pytest
from devutil import free_port

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    for sub in ("", "oracle", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    from devutil import HostOps, ScheduleHandle, ShmIpc
    from dgt.dist import HostClock, summa_benchmark

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r = summa_benchmark(150, 170, 90, 16, 24, 20, steps=2, warmup=1, alpha=1.5, beta=-0.5, ops=HostOps(),
                            ipc=ShmIpc(), handle=ScheduleHandle(), clock=HostClock(), device="cpu", seed=3)
        out.put((rank, r))
        dist.barrier()
    except Exception:
        import traceback

        out.put((rank, traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,grid", [(4, [2, 2]), (2, [2, 1])])
def test_summa_benchmark_gloo(world, grid):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    results = {}
    for _ in range(world):
        rank, r = out.get(timeout=180)
        if isinstance(r, str):
            for pr in procs:
                pr.join(timeout=30)
            pytest.fail(f"rank {rank} failed:\n{r}")
        results[rank] = r
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    r0 = results[0]
    assert r0["grid"] == grid and r0["ranks"] == world
    for form in ("collective", "fused"):
        assert r0[form]["ms"] > 0 and r0[form]["tflops"] > 0 and r0[form]["compute_ms"] > 0
        assert all(results[r][form]["ms"] == r0[form]["ms"] for r in results)  # the max over ranks
    assert r0["fused_vs_collective_rel"] <= 1e-13
