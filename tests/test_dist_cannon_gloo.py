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


def _driver_rank(rank, p, c, fused, log_dir, port, out):
    import datetime

    import torch.distributed as dist

    for sub in ("", "oracle", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    from devutil import CannonHandle, HostOps, ShmIpc
    from dgt.dist import pre_distributed_cannon25_nccl

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=p * p * c, timeout=datetime.timedelta(seconds=60))
    try:
        kw = dict(ipc=ShmIpc(), handle=CannonHandle()) if fused else dict(ops=HostOps())
        C = pre_distributed_cannon25_nccl(p, c, 40, 2, alpha=1.5, beta=-0.5, gather_results=True, log_dir=log_dir,
                                          machine="b200test", fused=fused, seed=5, sync=lambda: None, **kw)
        if rank == 0:
            out.put((rank, C))
        dist.barrier()
    except Exception:
        import traceback

        out.put((-1, traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("p,c,fused", [(2, 1, False), (2, 2, True)])
def test_nccl_driver_log_and_result(p, c, fused, tmp_path):
    """pre_distributed_cannon25_nccl (the reference's preDistributedCannon25NCCL) on gloo
    ranks: rank 0 gathers C after two runs (C <- alpha A B + beta C each run) and appends
    one row per run in the reference's NCCL schema."""
    import torch.multiprocessing as mp

    pd = pytest.importorskip("pandas")
    sys.path.insert(0, os.path.join(ROOT, "distributed-gemm-thesis_b200"))
    from dgt import csvlog

    world = p * p * c
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_driver_rank, args=(r, p, c, fused, str(tmp_path), port, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    rank, C = out.get(timeout=180)
    for pr in procs:
        pr.join(timeout=60)
    assert rank == 0, C
    assert all(pr.exitcode == 0 for pr in procs)
    rng = np.random.Generator(np.random.PCG64(5))
    A, B, C0 = (rng.uniform(-1.0, 1.0, (40, 40)) for _ in range(3))
    AB = A @ B
    want = 1.5 * AB + -0.5 * (1.5 * AB + -0.5 * C0)
    assert np.abs(C - want).max() <= 1e-12
    path = tmp_path / csvlog.cannon_nccl_log_name("b200test")
    assert path.name == "DGEMM_execution_logs-PreDistributed_GEMM-b200test-2.5DCANNON-dgt-NCCL.csv"
    df = pd.read_csv(path, header=0)
    assert list(df.columns) == csvlog.CANNON_NCCL_HEADER.split(",")
    assert len(df) == 2 and (df["TotalGPUs"] == world).all() and (df["StackSize"] == c).all()
    assert (df["Algo"] == ("2.5D CANNON dgt peer" if fused else "2.5D CANNON dgt NCCL")).all()


def test_csvlog_rules(tmp_path):
    """The Python log helpers keep the reference's rules: header once, a foreign first line
    gets the header appended, %lf-style rows."""
    sys.path.insert(0, os.path.join(ROOT, "distributed-gemm-thesis_b200"))
    from dgt import csvlog

    row = csvlog.cannon_nccl_row("2.5D CANNON dgt NCCL", 8192, 8192, 8192, 1, 32, 4, 4, 2, 0.5, 0.03125, 0.125,
                                 csvlog.calculate_gflops(8192, 8192, 8192, 0.03125))
    assert row == "2.5D CANNON dgt NCCL,8192,8192,8192,1,32,4,4,2,0.500000,0.031250,0.125000,35184.372089,devices\n"
    path = tmp_path / "log.csv"
    for _ in range(2):
        f = csvlog.create_log_csv(str(path), csvlog.CANNON_NCCL_HEADER)
        csvlog.write_line_to_file(f, row)
        f.close()
    assert path.read_text() == csvlog.CANNON_NCCL_HEADER + "\n" + row + row
    other = tmp_path / "other.csv"
    other.write_text("Algo,M\nx,1\n")
    csvlog.create_log_csv(str(other), csvlog.CANNON_NCCL_HEADER).close()
    assert other.read_text() == "Algo,M\nx,1\n" + csvlog.CANNON_NCCL_HEADER + "\n"
