"""SUMMA across processes (dgt.dist.DistSumma) as four gloo ranks on the CPU: the step
schedule -- panel owners, row and column broadcasts on the process-grid sub-groups, the
ragged last panel, beta applied once, lookahead buffers -- with a host double standing in
for the rank-local operations (on a GPU they are dgt_dgemm and dgt_copy_block).  Each rank
starts from its block-cyclic locals (a scatter that equals the oracle's, which is pinned to
the reference's pblasDecomposer, and that also covers grids leaving a process row empty);
the gathered C must equal the host FP64 GEMM within 1e-13 (relative Frobenius; summation
order differs)."""
import os
import socket
import sys

import numpy as np
import pytest
from devutil import free_port, gather_block_cyclic, local_tensor, scatter_block_cyclic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (p, q, mb, nb, kb, M, N, K, alpha, beta)
CASES = [
    (2, 2, 16, 24, 20, 150, 170, 90, 1.5, -0.5),   # ragged everywhere, 5 panels (last 10 wide)
    (1, 4, 32, 16, 8, 64, 100, 77, 1.0, 0.0),      # one process row: no column broadcasts
    (4, 1, 16, 32, 12, 40, 50, 61, -2.0, 1.0),     # process row 3 owns no rows of A or C
    (2, 2, 16, 16, 16, 48, 40, 0, 1.0, 0.25),      # K = 0: C = beta C
]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    for sub in ("", "oracle", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import oracle as O
    from devutil import HostOps
    from dgt.dist import DistSumma

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        for n_case, (p, q, mb, nb, kb, M, N, K, alpha, beta) in enumerate(CASES):
            A, B, C = (O.uniform(shape, 10 * n_case + s) for s, shape in ((1, (M, K)), (2, (K, N)), (3, (M, N))))
            la = scatter_block_cyclic(A, mb, kb, p, q)[rank]
            lb = scatter_block_cyclic(B, kb, nb, p, q)[rank]
            lc = scatter_block_cyclic(C, mb, nb, p, q)[rank]
            tA, tB, tC = local_tensor(la), local_tensor(lb), local_tensor(lc)
            S = DistSumma(p, q, mb, nb, kb, ops=HostOps())
            assert S.local_shapes(M, N, K) == (la.shape, lb.shape, lc.shape)
            S.multiply(M, N, K, alpha, tA, tB, beta, tC)
            rows, cols = lc.shape
            got = tC.numpy()[:cols, :rows].T.copy() if rows and cols else np.zeros((rows, cols))
            out.put((n_case, rank, got))
        dist.barrier()
    except Exception:
        import traceback

        out.put((-1, rank, traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


def test_dist_summa_four_gloo_ranks():
    import torch.multiprocessing as mp

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

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
        assert O.rel_errors(G, ref)[1] <= 1e-13, (n_case, O.rel_errors(G, ref))


def test_scatter_helper_matches_oracle():
    """The test's block-cyclic scatter equals the oracle's (pinned to the reference's
    pblasDecomposer) wherever the oracle accepts the grid, and gather inverts it."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    for (M, N, mb, nb, p, q) in [(150, 90, 16, 20, 2, 2), (64, 77, 32, 8, 1, 4), (170, 61, 24, 12, 4, 1)]:
        G = O.uniform((M, N), M)
        mine = scatter_block_cyclic(G, mb, nb, p, q)
        for a, b in zip(mine, O.orc().pblas_scatter(G, mb, nb, p, q)):
            assert np.array_equal(a, b)
        assert np.array_equal(gather_block_cyclic(mine, M, N, mb, nb, p, q), G)
    G = O.uniform((40, 50), 1)
    assert scatter_block_cyclic(G, 16, 32, 4, 1)[3].shape == (0, 50)  # a process row without rows


def test_dist_summa_needs_matching_world():
    """Outside an initialised process group, construction fails."""
    sys.path.insert(0, os.path.join(ROOT, "distributed-gemm-thesis_b200"))
    from dgt.dist import DistSumma

    with pytest.raises(RuntimeError):
        DistSumma(2, 2, 16, 16, 16)


class _PtrHandle:
    """dgt.Handle's copy_block and dgemm acting on host addresses, so DgtOps's pointer and
    leading-dimension arithmetic runs unchanged on CPU tensors."""

    @staticmethod
    def _mat(addr, rows, cols, ld):
        import ctypes

        n = ld * (cols - 1) + rows if rows and cols else 0
        buf = np.frombuffer((ctypes.c_double * max(n, 1)).from_address(addr), dtype=np.float64)
        return np.lib.stride_tricks.as_strided(buf, shape=(rows, cols), strides=(8, 8 * ld))

    def copy_block(self, rows, cols, src, dst, ldS, ldD, col_major=True):
        assert col_major and ldS >= rows and ldD >= rows
        self._mat(dst, rows, cols, ldD)[...] = self._mat(src, rows, cols, ldS)

    def dgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, mode=None, slices=7):
        assert ta == tb == "N" and lda >= max(1, m) and ldb >= max(1, k) and ldc >= max(1, m)
        c = self._mat(C, m, n, ldc)
        prod = self._mat(A, m, k, lda) @ self._mat(B, k, n, ldb) if k else 0.0
        c[...] = alpha * prod if beta == 0.0 else alpha * prod + beta * c


def test_device_ops_argument_arithmetic():
    """DistSumma on a 1 x 1 grid (one-rank gloo group) through DgtOps -- the product's
    pointer offsets, leading dimensions and beta-on-the-first-panel rule -- with the handle
    replaced by a host-address double."""
    import datetime

    import torch
    import torch.distributed as dist

    for sub in ("oracle", "distributed-gemm-thesis_b200"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import oracle as O
    from dgt.dist import DgtOps, DistCannon25D, DistSumma

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        M, N, K = 70, 50, 45
        A, B, C = O.uniform((M, K), 4), O.uniform((K, N), 5), O.uniform((M, N), 6)
        tA, tB, tC = (local_tensor(x) for x in (A, B, C))
        DistSumma(1, 1, 16, 16, 8, ops=DgtOps(_PtrHandle())).multiply(M, N, K, 1.5, tA, tB, -0.5, tC)
        got = tC.numpy().T
        assert O.rel_errors(got, O.dgemm(A, B, 1.5, -0.5, C))[1] <= 1e-13
        S = O.uniform((40, 40), 7)
        tS, tT, tU = local_tensor(S), local_tensor(S.T.copy()), local_tensor(S)
        DistCannon25D(1, 1, ops=DgtOps(_PtrHandle())).multiply(40, 2.0, tS, tT, 0.5, tU)
        assert O.rel_errors(tU.numpy().T, O.dgemm(S, S.T, 2.0, 0.5, S))[1] <= 1e-13
        dst = torch.zeros_like(tS)
        DgtOps(_PtrHandle()).copy(tS, dst)  # the skew's copy of a tile that stays put
        assert torch.equal(dst, tS)
    finally:
        dist.destroy_process_group()


def _dying_rank_main(rank, port, out):
    import datetime

    import torch.distributed as dist

    for sub in ("", "oracle", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import oracle as O
    from devutil import HostOps
    from dgt.dist import DistSumma

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=4, timeout=datetime.timedelta(seconds=10))
    p, q, b, M, N, K = 2, 2, 16, 64, 64, 64
    A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
    tA, tB, tC = (local_tensor(scatter_block_cyclic(X, b, b, p, q)[rank]) for X in (A, B, C))
    S = DistSumma(p, q, b, b, b, ops=HostOps())
    if rank == 3:
        os._exit(1)  # leaves between steps: none of its collectives is in flight
    try:
        S.multiply(M, N, K, 1.0, tA, tB, 0.0, tC)
        out.put((rank, "finished"))
    except Exception:
        out.put((rank, "error"))


def test_dist_summa_rank_failure_ends_in_errors_not_a_hang():
    """A rank that exits before the step loop: every other rank's step loop ends with an
    error instead of waiting for ever -- the ranks sharing its process row or column at their
    next broadcast (gloo notices the closed connection, or the 10 s group timeout ends the
    wait), and rank 0, which shares no group with it, once those ranks have left its own
    row and column broadcasts in turn."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_dying_rank_main, args=(r, port, out)) for r in range(4)]
    for pr in procs:
        pr.start()
    got = dict(out.get(timeout=120) for _ in range(3))
    for pr in procs:
        pr.join(timeout=60)
    assert got == {0: "error", 1: "error", 2: "error"}
    assert procs[3].exitcode == 1
