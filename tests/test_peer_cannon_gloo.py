"""2.5D Cannon with its communication fused into the kernels (dgt.dist.PeerCannon25D) as
gloo ranks on the CPU, with process-shared memory standing in for CUDA IPC.  A handle
double runs on those addresses what dgt_cannon25d_rank's kernel runs -- the k-block order
dgt_cannon_schedule reports, each block read from its owner's tile -- and what
dgt_reduce_tiles runs -- the other stacks' partials added in stack order, read from their
ranks.  Grids 2x2x1, 2x2x2 and 3x3x1 (where the reference's rotations skip k-blocks and the
shift-by-one order is used); the partial buffers of stacks above 0 start as NaN, so any
read of an unwritten partial would show.  Stack 0's tiles must equal the host FP64 GEMM
within 1e-13 (relative Frobenius)."""
import os
import socket
import sys

import numpy as np
import pytest
from devutil import CannonHandle, free_port

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, p, c, M, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    for sub in ("", "oracle", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import oracle as O
    from dgt.dist import PeerCannon25D
    from devutil import ShmIpc

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=p * p * c, timeout=datetime.timedelta(seconds=60))
    try:
        lm = M // p
        k, i, j = rank // (p * p), (rank // p) % p, rank % p
        A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
        tile = lambda X: torch.from_numpy(np.ascontiguousarray(X[i * lm:(i + 1) * lm, j * lm:(j + 1) * lm].T))
        ipc = ShmIpc()
        S = PeerCannon25D(p, c, M, ipc=ipc, handle=CannonHandle())
        C_tile = None
        if k == 0:
            S.A_tile.copy_(tile(A))
            S.B_tile.copy_(tile(B))
            C_tile = tile(C).clone()
        else:
            ipc.tensor(S._partial, (lm, lm)).fill_(float("nan"))
        S.multiply(1.5, -0.5, C_tile)
        if k == 0:
            out.put((rank, C_tile.numpy().T.copy()))
        S.close()
    except Exception:
        import traceback

        out.put((-1, traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("p,c,M", [(2, 1, 48), (2, 2, 40), (3, 1, 45)])
def test_peer_cannon_gloo(p, c, M):
    import torch.multiprocessing as mp

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    world = p * p * c
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, p, c, M, port, out)) for r in range(world)]
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
        G[(r // p) * lm:(r // p + 1) * lm, (r % p) * lm:(r % p + 1) * lm] = t
    A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
    assert O.rel_errors(G, O.dgemm(A, B, 1.5, -0.5, C))[1] <= 1e-13
