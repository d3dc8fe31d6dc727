"""2.5D Cannon across processes (dgt.dist.DistCannon25D) as gloo ranks on the CPU: stack
broadcast, skew, unit shifts with the next shift posted before each GEMM, and the stack
reduction, with a host double for the rank-local GEMM (dgt_dgemm on a GPU).  Grids: 2x2x1
(world 4), 2x2x2 (world 8: broadcast and reduce, no shifts) and 3x3x1 (world 9, where the
reference's growing rotations skip k-blocks).  Stacks above 0 start from C tiles of NaN,
which must never be read.  The assembled stack-0 C must equal the host FP64 GEMM within
1e-13 (relative Frobenius)."""
import os
import socket
import sys

import numpy as np
import pytest
from devutil import free_port

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _tile(X, i, j, lm):
    import torch

    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(X[i * lm:(i + 1) * lm, j * lm:(j + 1) * lm]).T))


def _rank_main(rank, p, c, M, alpha, beta, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    for sub in ("", "oracle", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import oracle as O
    from devutil import HostOps
    from dgt.dist import DistCannon25D

    world = p * p * c
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
        lm = M // p
        k, i, j = rank // (p * p), (rank // p) % p, rank % p
        if k == 0:
            tA, tB, tC = _tile(A, i, j, lm), _tile(B, i, j, lm), _tile(C, i, j, lm)
        else:
            tA, tB, tC = (torch.full((lm, lm), float("nan"), dtype=torch.float64) for _ in range(3))
        a_in, b_in = tA.clone(), tB.clone()
        S = DistCannon25D(p, c, ops=HostOps())
        S.multiply(M, alpha, tA, tB, beta, tC)
        if k == 0:
            # the caller's A and B tiles are not shifted in place
            assert torch.equal(tA, a_in) and torch.equal(tB, b_in)
            out.put((rank, tC.numpy().T.copy()))
        dist.barrier()
    except Exception:
        import traceback

        out.put((-1, traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("p,c,M", [(2, 1, 48), (2, 2, 40), (3, 1, 45)])
def test_dist_cannon_gloo(p, c, M):
    import torch.multiprocessing as mp

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    alpha, beta = 1.5, -0.5
    world = p * p * c
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, p, c, M, alpha, beta, port, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    tiles = {}
    for _ in range(p * p):
        rank, got = out.get(timeout=180)
        if rank < 0:
            for pr in procs:
                pr.join(timeout=30)
            pytest.fail(got)
        tiles[rank] = got
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    lm = M // p
    G = np.zeros((M, M))
    for r, t in tiles.items():
        i, j = r // p, r % p
        G[i * lm:(i + 1) * lm, j * lm:(j + 1) * lm] = t
    A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
    assert O.rel_errors(G, O.dgemm(A, B, alpha, beta, C))[1] <= 1e-13
