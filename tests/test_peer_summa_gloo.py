"""SUMMA with the broadcasts fused into the GEMM (dgt.dist.PeerSumma) as four gloo ranks on
the CPU.  Process-shared memory (multiprocessing.shared_memory) stands in for CUDA IPC, and
a handle double runs, on those addresses, exactly the K segments dgt_summa_schedule gives
each rank -- the segment list dgt_summa_rank's kernel walks.  So the test exercises the
whole host side of the fused path across real processes: buffer sizes, handle exchange,
the peer pointer arrays, the barriers, and each rank reading its panels straight out of the
owners' memory.  The gathered C must equal the host FP64 GEMM within 1e-13."""
import os
import socket
import sys

import numpy as np
import pytest
from devutil import ScheduleHandle, ShmIpc, free_port

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = [  # (p, q, mb, nb, kb, M, N, K, alpha, beta)
    (2, 2, 16, 24, 20, 150, 170, 90, 1.5, -0.5),
    (1, 4, 32, 16, 8, 64, 100, 77, 1.0, 0.0),
    (4, 1, 16, 32, 12, 40, 50, 61, -2.0, 1.0),  # process row 3 owns no rows of A or C
    (2, 2, 16, 16, 16, 48, 40, 0, 1.0, 0.25),   # K = 0: C = beta C
]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    for sub in ("", "oracle", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import oracle as O
    from dgt.dist import PeerSumma
    from devutil import local_tensor, scatter_block_cyclic

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        for n_case, (p, q, mb, nb, kb, M, N, K, alpha, beta) in enumerate(CASES):
            A, B, C = (O.uniform(shape, 10 * n_case + s) for s, shape in ((1, (M, K)), (2, (K, N)), (3, (M, N))))
            S = PeerSumma(p, q, mb, nb, kb, M, N, K, ipc=ShmIpc(), handle=ScheduleHandle())
            la, lb, lc = (scatter_block_cyclic(X, r, c, p, q)[rank] for X, r, c in ((A, mb, kb), (B, kb, nb), (C, mb, nb)))
            S.A_loc.copy_(local_tensor(la))
            S.B_loc.copy_(local_tensor(lb))
            tC = local_tensor(lc)
            S.multiply(alpha, beta, tC)
            # the owners' A and B are untouched by the peers' reads
            assert torch.equal(S.A_loc, local_tensor(la)) and torch.equal(S.B_loc, local_tensor(lb))
            rows, cols = lc.shape
            out.put((n_case, rank, tC.numpy()[:cols, :rows].T.copy()))
            S.close()
        dist.barrier()
    except Exception:
        import traceback

        out.put((-1, rank, traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


def test_peer_summa_four_gloo_ranks():
    import torch.multiprocessing as mp

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    from devutil import gather_block_cyclic

    world = 4
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    results = {}
    for _ in range(world * len(CASES)):
        n_case, rank, got = out.get(timeout=180)
        if n_case < 0:
            for pr in procs:
                pr.join(timeout=30)
            pytest.fail(f"rank {rank} failed:\n{got}")
        results[(n_case, rank)] = got
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for n_case, (p, q, mb, nb, kb, M, N, K, alpha, beta) in enumerate(CASES):
        A, B, C = (O.uniform(shape, 10 * n_case + s) for s, shape in ((1, (M, K)), (2, (K, N)), (3, (M, N))))
        G = gather_block_cyclic([results[(n_case, r)] for r in range(world)], M, N, mb, nb, p, q)
        ref = O.dgemm(A, B, alpha, beta, C) if K > 0 else beta * C
        assert O.rel_errors(G, ref)[1] <= 1e-13, n_case


class _FailingOpenIpc(ShmIpc):
    def __init__(self):
        super().__init__()
        self.freed = []

    def open(self, handle):
        raise RuntimeError("mapping refused")

    def free(self, ptr):
        self.freed.append(ptr)  # unlinked after the barrier: the peer may still be mapping it


def _failing_rank(rank, port, out):
    import datetime

    import torch.distributed as dist

    for sub in ("", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    from dgt.dist import PeerSumma

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
    try:
        ipc = _FailingOpenIpc() if rank == 1 else ShmIpc()
        own = []
        try:
            S = PeerSumma(1, 2, 16, 16, 16, 32, 32, 32, ipc=ipc, handle=ScheduleHandle())
            own = [ptr for ptr, _ in S._own]
            out.put((rank, "built", len(S.A_ptrs)))
        except RuntimeError as e:
            out.put((rank, str(e), len(ipc.freed)))
        dist.barrier()
        for ptr in own + getattr(ipc, "freed", []):
            ShmIpc.free(ipc, ptr)
    finally:
        dist.destroy_process_group()


def test_peer_summa_setup_failure_releases_buffers():
    """A rank that cannot map a peer's buffer raises, after freeing the two buffers it
    allocated; the group is still usable (a barrier completes)."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_failing_rank, args=(r, port, out)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = dict((r, (msg, n)) for r, msg, n in (out.get(timeout=120) for _ in procs))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert got[0] == ("built", 2)
    assert got[1] == ("mapping refused", 2)
