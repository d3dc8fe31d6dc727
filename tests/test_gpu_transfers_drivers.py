"""GPU checks of the transfers at the edges of the hot path, through the C ABI:
 * the block-cyclic scatter / gather with the global matrix in page-locked host memory
   (dgt_pack_block_cyclic_host / dgt_unpack_block_cyclic_host), bit-exact against the
   device-global entry points on the same inputs, and pageable memory refused;
 * copyBlock<float> (dgt_copy_block_f32), bit-exact;
 * the reference-shaped 2.5D Cannon benchmark drivers and their CSV logs
   (include/dgt_drivers.hpp, tests/cpp/driver_test.cpp);
 * SUMMA across processes (dgt.dist) with its device operations (dgt_copy_block panel
   packing, dgt_dgemm steps) on one rank;
 * one rank's share of the SUMMA (dgt_summa_rank), the form a multi-GPU run uses with other
   GPUs' buffers in its pointer arrays, against the whole-grid dgt_summa;
 * PeerSumma over CUDA IPC buffers (dgt_ipc_*): one process, and two processes sharing the
   GPU that read each other's panels;
 * the benchmark command line (bin/dgt_cublas25d_benchmark) with its CSV rows;
 * the 2.5D Cannon per rank (dgt_cannon25d_rank + dgt_reduce_tiles) against the in-device
   dgt_cannon25d, and PeerCannon25D as eight processes sharing the GPU;
 * guard bands around dgt_dgemm's operands in every FP64 mode (nothing written outside C)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import dgt
import oracle as O
from devutil import check_cannon_driver_logs, dev, host, ptr

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def h():
    with dgt.Handle() as handle:
        yield handle


def _pinned_global(G, ldg, fill):
    """Column-major M x N matrix G in a page-locked host buffer with leading dimension ldg
    (rows M..ldg-1 of every column hold `fill`), as a torch tensor and its address."""
    import torch

    M, N = G.shape
    buf = np.full((N, ldg), fill, dtype=np.float64)
    buf[:, :M] = G.T
    t = torch.from_numpy(buf).pin_memory()
    return t, t.data_ptr()


def _locals(M, N, mb, nb, p, q):
    import torch

    rows = [dgt.numroc(M, mb, r // q, 0, p) for r in range(p * q)]
    cols = [dgt.numroc(N, nb, r % q, 0, q) for r in range(p * q)]
    lld = [max(x, 1) for x in rows]
    locs = [torch.full((max(c, 1), l), -3.0, dtype=torch.float64, device="cuda") for c, l in zip(cols, lld)]
    return locs, lld


@pytest.mark.parametrize("M,N,mb,nb,p,q,ldg", [(300, 250, 32, 24, 2, 3, 300), (517, 389, 64, 64, 4, 4, 530),
                                               (40, 70, 64, 16, 3, 2, 41)])
def test_block_cyclic_from_host_equals_device_path(h, M, N, mb, nb, p, q, ldg):
    import torch

    G = O.uniform((M, N), M + N)
    tG, pG = _pinned_global(G, ldg, 7.0)
    # device path on the same matrix
    dG = dev(np.asfortranarray(tG.numpy().T))  # ldg x N, column-major
    want, lld = _locals(M, N, mb, nb, p, q)
    h.pack_block_cyclic(M, N, mb, nb, p, q, ptr(dG), ldg, [ptr(t) for t in want], lld)
    got, _ = _locals(M, N, mb, nb, p, q)
    h.pack_block_cyclic_host(M, N, mb, nb, p, q, pG, ldg, [ptr(t) for t in got], lld)
    torch.cuda.synchronize()
    h.check_device()
    for a, b in zip(got, want):
        assert torch.equal(a.view(torch.int64), b.view(torch.int64))
    # gather back into a second pinned buffer: the matrix, padding rows untouched
    tB, pB = _pinned_global(np.zeros((M, N)), ldg, -9.0)
    h.unpack_block_cyclic_host(M, N, mb, nb, p, q, pB, ldg, [ptr(t) for t in got], lld)
    torch.cuda.synchronize()
    h.check_device()
    back = tB.numpy()
    assert np.array_equal(back[:, :M].T, G)
    assert (back[:, M:] == -9.0).all()


def test_block_cyclic_host_refuses_pageable(h):
    M, N, mb, nb, p, q = 64, 48, 16, 16, 2, 2
    G = np.asfortranarray(O.uniform((M, N), 3))
    locs, lld = _locals(M, N, mb, nb, p, q)
    with pytest.raises(dgt.DgtError) as e:
        h.pack_block_cyclic_host(M, N, mb, nb, p, q, G.ctypes.data, M, [ptr(t) for t in locs], lld)
    assert e.value.status == 1
    with pytest.raises(dgt.DgtError) as e:
        h.unpack_block_cyclic_host(M, N, mb, nb, p, q, G.ctypes.data, M, [ptr(t) for t in locs], lld)
    assert e.value.status == 1


# (rows, cols, ldS, ldD, source offset, destination offset in floats, column-major): the
# offsets put the runs in every 16-byte phase, same and different on the two sides, so the
# head / float4 body / tail split and the scalar path are all exercised.
@pytest.mark.parametrize("rows,cols,ldS,ldD,so,do_,cm", [
    (5, 7, 9, 6, 0, 0, True), (67, 5, 70, 68, 1, 3, True), (129, 4, 131, 133, 2, 2, True),
    (3, 300, 3, 5, 1, 1, True), (64, 3, 64, 64, 3, 3, True), (3, 64, 70, 65, 0, 2, False),
    (1, 1, 1, 1, 0, 0, True), (1031, 2, 1033, 1037, 1, 1, True), (2, 2, 2, 2, 3, 3, True),
])
def test_copy_block_f32(h, rows, cols, ldS, ldD, so, do_, cm):
    """copyBlock<float>: bit-exact strided copy, the destination's other elements untouched."""
    import torch

    r, c = (rows, cols) if cm else (cols, rows)
    rng = np.random.default_rng(rows * 7 + cols)
    src = rng.standard_normal(so + ldS * c).astype(np.float32)
    dst0 = rng.standard_normal(do_ + ldD * c).astype(np.float32)
    ds, dd = torch.from_numpy(src).cuda(), torch.from_numpy(dst0.copy()).cuda()
    h.copy_block_f32(rows, cols, ptr(ds) + 4 * so, ptr(dd) + 4 * do_, ldS, ldD, cm)
    torch.cuda.synchronize()
    h.check_device()
    want = dst0.copy()
    for j in range(c):
        want[do_ + j * ldD:do_ + j * ldD + r] = src[so + j * ldS:so + j * ldS + r]
    assert np.array_equal(dd.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_copy_block_f32_rejects_bad_arguments(h):
    """Host-side checks, before any launch: misaligned pointer, short leading dimension."""
    import torch

    x = torch.zeros(64, dtype=torch.float32, device="cuda")
    with pytest.raises(dgt.DgtError) as e:
        h.copy_block_f32(4, 4, ptr(x) + 2, ptr(x) + 32, 4, 4)
    assert e.value.status == 1
    with pytest.raises(dgt.DgtError) as e:
        h.copy_block_f32(8, 2, ptr(x), ptr(x) + 128, 4, 8)
    assert e.value.status == 1
    h.copy_block_f32(0, 5, ptr(x), ptr(x), 1, 1)  # empty: no launch, no error


def test_cpp_cannon_drivers_and_logs(tmp_path):
    """include/dgt_drivers.hpp: fullOffloadSumma25Dgemm / preDistributedSumma25Dgemm results
    against host triple loops (tests/cpp/driver_test.cpp), then their CSV rows read back
    the way the thesis notebooks read them."""
    lib = os.path.join(ROOT, "distributed-gemm-thesis_b200", "lib")
    exe = str(tmp_path / "driver_test")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "driver_test.cpp"),
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"), "-L", lib, "-ldgt",
                    "-L", os.path.join(cuda, "lib64"), "-lcudart", f"-Wl,-rpath,{lib}", "-o", exe], check=True)
    logs = tmp_path / "logs"
    logs.mkdir()
    out = subprocess.run([exe, str(logs)], capture_output=True, text=True, timeout=300)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ALL OK" in out.stdout

    check_cannon_driver_logs(logs)


def test_dist_summa_device_ops_one_rank():
    """dgt.dist.DistSumma on a 1 x 1 grid (a one-rank gloo group, so no collective runs):
    every K panel goes through DgtOps -- B's panel rows packed by dgt_copy_block, the step
    GEMM by dgt_dgemm with beta on the first panel only -- against the host FP64 GEMM."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist
    from dgt.dist import DistSumma

    M, N, K, kb = 300, 200, 170, 32  # 6 panels, the last 10 wide
    A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        tA, tB, tC = dev(A), dev(B), dev(C)  # (cols, rows) tensors: column-major, ld = rows
        S = DistSumma(1, 1, 64, 64, kb)
        S.multiply(M, N, K, 1.5, tA, tB, -0.5, tC)
        torch.cuda.synchronize()
        S.ops.h.check_device()
        got = np.asfortranarray(tC.cpu().numpy().T)
    finally:
        dist.destroy_process_group()
    assert O.rel_errors(got, O.dgemm(A, B, 1.5, -0.5, C))[1] <= 1e-13


@pytest.mark.parametrize("M,N,K,b,p,q", [(257, 131, 199, 32, 2, 3), (500, 400, 300, 64, 4, 4)])
def test_summa_rank_matches_whole_grid(h, M, N, K, b, p, q):
    """Every rank's dgt_summa_rank equals its block of the whole-grid dgt_summa (same
    segments, same kernel; relative Frobenius <= 1e-14), and the assembled result the host
    FP64 GEMM (<= 1e-13)."""
    import torch

    A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
    o = O.orc()

    def pack(X, rows, cols):
        shapes = o.pblas_shapes(rows, cols, b, b, p, q)
        locs = [torch.zeros((max(c, 1), max(r, 1)), dtype=torch.float64, device="cuda") for r, c, _ in shapes]
        lld = [max(r, 1) for r, _, _ in shapes]
        dX = dev(X)
        h.pack_block_cyclic(rows, cols, b, b, p, q, ptr(dX), rows, [ptr(l) for l in locs], lld)
        return dX, locs, lld

    _, lA, lldA = pack(A, M, K)
    _, lB, lldB = pack(B, K, N)
    dC, lC, lldC = pack(C, M, N)
    lC_rank = [x.clone() for x in lC]
    pA, pB = [ptr(x) for x in lA], [ptr(x) for x in lB]
    h.summa(p, q, b, b, b, M, N, K, 1.5, pA, lldA, pB, lldB, -0.5, [ptr(x) for x in lC], lldC)
    for r in range(p * q):
        h.summa_rank(r, p, q, b, b, b, M, N, K, 1.5, pA, lldA, pB, lldB, -0.5, ptr(lC_rank[r]), lldC[r])
    torch.cuda.synchronize()
    h.check_device()
    for r in range(p * q):
        whole, mine = lC[r].cpu().numpy(), lC_rank[r].cpu().numpy()
        assert O.rel_errors(mine, whole)[1] <= 1e-14, r
    h.unpack_block_cyclic(M, N, b, b, p, q, ptr(dC), M, [ptr(x) for x in lC_rank], lldC)
    torch.cuda.synchronize()
    assert O.rel_errors(host(dC, (M, N)), O.dgemm(A, B, 1.5, -0.5, C))[1] <= 1e-13


def _peer_rank(rank, world, p, q, port, out):
    """One rank of PeerSumma over real CUDA IPC (every rank on cuda:0)."""
    import datetime

    import torch
    import torch.distributed as dist

    for sub in ("", "oracle", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import oracle as O
    from dgt.dist import PeerSumma
    from devutil import local_tensor, scatter_block_cyclic

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        M, N, K, mb, nb, kb = 300, 260, 170, 32, 48, 40
        A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
        S = PeerSumma(p, q, mb, nb, kb, M, N, K)
        la, lb, lc = (scatter_block_cyclic(X, r, c, p, q)[rank] for X, r, c in ((A, mb, kb), (B, kb, nb), (C, mb, nb)))
        S.A_loc.copy_(local_tensor(la).cuda())
        S.B_loc.copy_(local_tensor(lb).cuda())
        tC = local_tensor(lc).cuda()
        S.multiply(1.5, -0.5, tC)
        S.h.check_device()
        rows, cols = lc.shape
        out.put((rank, tC.cpu().numpy()[:cols, :rows].T.copy()))
        S.close()
    except Exception:
        import traceback

        out.put((-1, traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


def _run_peer(world, p, q):
    import socket

    import torch.multiprocessing as mp
    from devutil import gather_block_cyclic

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_peer_rank, args=(r, world, p, q, port, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = {}
    for _ in range(world):
        rank, res = out.get(timeout=300)
        if rank < 0:
            for pr in procs:
                pr.join(timeout=60)
            pytest.fail(res)
        got[rank] = res
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    M, N, K, mb, nb, kb = 300, 260, 170, 32, 48, 40
    A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
    G = gather_block_cyclic([got[r] for r in range(world)], M, N, mb, nb, p, q)
    assert O.rel_errors(G, O.dgemm(A, B, 1.5, -0.5, C))[1] <= 1e-13


def test_peer_summa_one_process():
    """PeerSumma on a 1 x 1 grid: dgt_ipc_alloc buffers viewed as tensors, dgt_summa_rank on
    them, dgt_ipc_free."""
    _run_peer(1, 1, 1)


def test_peer_summa_two_processes_share_one_gpu():
    """Two processes on one GPU, each mapping the other's A and B through dgt_ipc_open: each
    rank's dgt_summa_rank reads its peer's panels directly.  The kernels only read data that
    host barriers have published; neither waits on the other."""
    _run_peer(2, 1, 2)


def test_benchmark_cli_on_gpu(tmp_path):
    """The built dgt_cublas25d_benchmark (the reference's cuBLAS25Benchmark command line):
    a pre-distributed run and a full-offload run append their CSV rows."""
    import pandas as pd

    exe = os.path.join(ROOT, "distributed-gemm-thesis_b200", "bin", "dgt_cublas25d_benchmark")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "distributed-gemm-thesis_b200")], check=True)
    for extra in ([], ["1"]):
        r = subprocess.run([exe, "NN", "512", "512", "512", "1.0", "0.0", "4", "4", "2", "2", "devices", *extra,
                            "--machine", "b200test", "--logdir", str(tmp_path)], capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
    for kind in ("PreDistributed", "FullOffload"):
        df = pd.read_csv(tmp_path / f"DGEMM_execution_logs-{kind}_GEMM-b200test-2.5DCANNON-dgt.csv", header=0)
        assert len(df) == 2 and (df["GFlops"] > 0).all() and (df["StackSize"] == 2).all()


def test_cannon_rank_and_reduce_match_in_device(h):
    """Every rank's dgt_cannon25d_rank (stack partials in separate buffers) followed by
    dgt_reduce_tiles into the stack-0 tiles equals the in-device dgt_cannon25d: same
    k-block order, same summation order (relative Frobenius <= 1e-14 per tile)."""
    import torch

    M, p, c = 512, 4, 2
    lm = M // p
    A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
    dA, dB, dC = dev(A), dev(B), dev(C)
    tiles = lambda: [torch.zeros((lm, lm), dtype=torch.float64, device="cuda") for _ in range(p * p)]
    tA, tB, tC = tiles(), tiles(), tiles()
    h.pack_cannon2d(M, p, ptr(dA), ptr(dB), ptr(dC), [ptr(x) for x in tA], [ptr(x) for x in tB],
                    [ptr(x) for x in tC])
    mine = [x.clone() for x in tC]
    partials = [torch.full((lm, lm), float("nan"), dtype=torch.float64, device="cuda") for _ in range(p * p * (c - 1))]
    pA, pB = [ptr(x) for x in tA], [ptr(x) for x in tB]
    h.cannon25d(M, p, c, 1.5, pA, pB, -0.5, [ptr(x) for x in tC])
    for rank in range(p * p * c):
        k, r = rank // (p * p), rank % (p * p)
        out = mine[r] if k == 0 else partials[(k - 1) * p * p + r]
        h.cannon25d_rank(M, p, c, rank, 1.5, pA, pB, -0.5, ptr(out))
    for r in range(p * p):
        h.reduce_tiles(ptr(mine[r]), [ptr(partials[(k - 1) * p * p + r]) for k in range(1, c)], lm * lm)
    torch.cuda.synchronize()
    h.check_device()
    for r in range(p * p):
        assert O.rel_errors(mine[r].cpu().numpy(), tC[r].cpu().numpy())[1] <= 1e-14, r


def _peer_cannon_rank(rank, p, c, M, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    for sub in ("", "oracle", "distributed-gemm-thesis_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import oracle as O
    from dgt.dist import PeerCannon25D

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=p * p * c, timeout=datetime.timedelta(seconds=180))
    try:
        torch.cuda.set_device(0)
        lm = M // p
        k, i, j = rank // (p * p), (rank // p) % p, rank % p
        A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
        tile = lambda X: torch.from_numpy(np.ascontiguousarray(X[i * lm:(i + 1) * lm, j * lm:(j + 1) * lm].T)).cuda()
        S = PeerCannon25D(p, c, M)
        C_tile = None
        if k == 0:
            S.A_tile.copy_(tile(A))
            S.B_tile.copy_(tile(B))
            C_tile = tile(C)
        S.multiply(1.5, -0.5, C_tile)
        S.h.check_device()
        if k == 0:
            out.put((rank, C_tile.cpu().numpy().T.copy()))
        S.close()
    except Exception:
        import traceback

        out.put((-1, traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


def test_peer_cannon_eight_processes_share_one_gpu():
    """PeerCannon25D on a 2 x 2 x 2 grid, eight processes on one GPU: tiles read from their
    owners through dgt_ipc_open, the stack-1 partials summed into stack 0 by reading them
    from their ranks.  Kernels only read data host barriers have published."""
    import socket

    import torch.multiprocessing as mp

    p, c, M = 2, 2, 256
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_peer_cannon_rank, args=(r, p, c, M, port, out)) for r in range(p * p * c)]
    for pr in procs:
        pr.start()
    tiles = {}
    for _ in range(p * p):
        rank, got = out.get(timeout=400)
        if rank < 0:
            for pr in procs:
                pr.join(timeout=60)
            pytest.fail(got)
        tiles[rank] = got
    for pr in procs:
        pr.join(timeout=180)
        assert pr.exitcode == 0
    lm = M // p
    G = np.zeros((M, M))
    for r, t in tiles.items():
        G[(r // p) * lm:(r // p + 1) * lm, (r % p) * lm:(r % p + 1) * lm] = t
    A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
    assert O.rel_errors(G, O.dgemm(A, B, 1.5, -0.5, C))[1] <= 1e-13


GUARD = 4096  # doubles of canary before and after every buffer (same allocation: a stray write cannot fault)
CANARY = np.array([0x7FF4DEADBEEF0001], dtype=np.uint64).view(np.float64)[0]  # a signalling-NaN bit pattern


def _guarded(X, ld):
    """Device buffer: GUARD canaries, X column-major with leading dimension ld (padding rows
    canary too), GUARD canaries.  Returns (tensor, pointer to X, host image of the buffer)."""
    import torch

    rows, cols = X.shape
    img = np.full(2 * GUARD + ld * max(cols, 1), CANARY)
    for j in range(cols):
        img[GUARD + j * ld:GUARD + j * ld + rows] = X[:, j]
    t = torch.from_numpy(img.copy()).cuda()
    return t, t.data_ptr() + 8 * GUARD, img


@pytest.mark.parametrize("mode,S", [(dgt.FP64_NATIVE, 7), (dgt.FP64_OZAKI_INT8, 7), (dgt.FP64_OZAKI2_INT8, 14)])
def test_gemm_guard_bands(h, mode, S):
    """dgt_dgemm writes C's m x n block and nothing else: the canaries around A, B and C and
    the padding rows of C (ldc > m) are bit for bit unchanged, A and B are not modified, and C
    matches the host FP64 GEMM -- for ragged, tiny and transposed shapes (the substitute for a
    memory sanitizer on this pool)."""
    import torch

    for m, n, k, ta, tb in [(257, 131, 199, "N", "N"), (1, 1, 1, "N", "N"), (7, 13, 5, "T", "N"),
                            (130, 129, 300, "N", "T"), (65, 33, 17, "T", "T")]:
        A = O.uniform((k, m) if ta == "T" else (m, k), m + 1)
        B = O.uniform((n, k) if tb == "T" else (k, n), n + 2)
        C = O.uniform((m, n), k + 3)
        lda, ldb, ldc = A.shape[0] + 3, B.shape[0] + 1, m + 5
        tA, pA, iA = _guarded(A, lda)
        tB, pB, iB = _guarded(B, ldb)
        tC, pC, iC = _guarded(C, ldc)
        h.dgemm(ta, tb, m, n, k, 1.5, pA, lda, pB, ldb, -0.5, pC, ldc, mode=mode, slices=S)
        torch.cuda.synchronize()
        h.check_device()
        for t, img in ((tA, iA), (tB, iB)):
            assert np.array_equal(t.cpu().numpy().view(np.uint64), img.view(np.uint64)), (m, n, k, ta, tb)
        got = tC.cpu().numpy()
        outside = np.ones(got.shape, dtype=bool)
        for j in range(n):
            outside[GUARD + j * ldc:GUARD + j * ldc + m] = False
        assert np.array_equal(got[outside].view(np.uint64), iC[outside].view(np.uint64)), (m, n, k, ta, tb)
        res = np.stack([got[GUARD + j * ldc:GUARD + j * ldc + m] for j in range(n)], axis=1)
        tol = 1e-13 if mode != dgt.FP64_OZAKI_INT8 else 1e-12
        assert O.rel_errors(res, O.dgemm(A, B, 1.5, -0.5, C, ta, tb))[1] <= tol, (m, n, k, ta, tb)


def _pinned_flat(x, order):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(np.asarray(x, order=order).ravel(order=order))).pin_memory()
    return t, t.data_ptr()


@pytest.mark.parametrize("M,N,K,P", [(13, 11, 5, 6), (333, 171, 80, 5)])
@pytest.mark.parametrize("cm", [True, False])
def test_block2d_from_host_equals_device_path(h, M, N, K, P, cm):
    """deliverMatrix / gatherResult with A, B, C in page-locked host memory: the same locals
    as the device-memory entries, bit for bit, and C restored by the gather."""
    import torch

    order = "F" if cm else "C"
    A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
    lA, lB, lC = O.orc().block2d_deliver(A, B, C, P, cm)
    (hA, pA), (hB, pB), (hC, pC) = (_pinned_flat(x, order) for x in (A, B, C))
    dA, dB, dC = hA.cuda(), hB.cuda(), hC.cuda()
    mk = lambda ls: [torch.zeros(x.size, dtype=torch.float64, device="cuda") for x in ls]
    oA, oB, oC, rA, rB, rC = mk(lA), mk(lB), mk(lC), mk(lA), mk(lB), mk(lC)
    ps = lambda ts: [ptr(t) for t in ts]
    h.pack_block2d_host(M, N, K, P, cm, pA, pB, pC, ps(oA), ps(oB), ps(oC))
    h.pack_block2d(M, N, K, P, cm, ptr(dA), ptr(dB), ptr(dC), ps(rA), ps(rB), ps(rC))
    back, pBk = _pinned_flat(np.zeros((M, N)), order)
    h.unpack_block2d_host(M, N, P, cm, pBk, ps(oC))
    torch.cuda.synchronize()
    h.check_device()
    for got, want in zip(oA + oB + oC, rA + rB + rC):
        assert torch.equal(got, want)
    assert torch.equal(back, hC)


@pytest.mark.parametrize("M,p", [(300, 3), (512, 4)])
def test_cannon2d_from_host_equals_device_path(h, M, p):
    """decompose2D / reorderMatrix with A, B, C in page-locked host memory (the full-offload
    driver's path): the same tiles as the device-memory entries, C restored, pageable
    memory refused."""
    import torch

    A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
    (hA, pA), (hB, pB), (hC, pC) = (_pinned_flat(x, "F") for x in (A, B, C))
    dA, dB, dC = hA.cuda(), hB.cuda(), hC.cuda()
    lm = M // p
    mk = lambda: [torch.zeros((lm, lm), dtype=torch.float64, device="cuda") for _ in range(p * p)]
    oA, oB, oC, rA, rB, rC = mk(), mk(), mk(), mk(), mk(), mk()
    ps = lambda ts: [ptr(t) for t in ts]
    h.pack_cannon2d_host(M, p, pA, pB, pC, ps(oA), ps(oB), ps(oC))
    h.pack_cannon2d(M, p, ptr(dA), ptr(dB), ptr(dC), ps(rA), ps(rB), ps(rC))
    back, pBk = _pinned_flat(np.zeros((M, M)), "F")
    h.unpack_cannon2d_host(M, p, pBk, ps(oC))
    torch.cuda.synchronize()
    h.check_device()
    for got, want in zip(oA + oB + oC, rA + rB + rC):
        assert torch.equal(got, want)
    assert torch.equal(back, hC)
    pageable = np.asfortranarray(A)
    with pytest.raises(dgt.DgtError) as e:
        h.pack_cannon2d_host(M, p, pageable.ctypes.data, pA, pC, ps(oA), ps(oB), ps(oC))
    assert e.value.status == dgt.INVALID_VALUE


def test_summa_guard_bands(h):
    """dgt_summa on a 2 x 3 grid with every rank's A, B and C local between canaries and
    padded leading dimensions: only the C blocks' valid rows change, and the gathered result
    is the host FP64 GEMM."""
    import torch

    from devutil import gather_block_cyclic, scatter_block_cyclic

    p, q, b, M, N, K = 2, 3, 32, 257, 131, 199
    A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
    la, lb, lc = (scatter_block_cyclic(X, b, b, p, q) for X in (A, B, C))
    gA = [_guarded(x, max(x.shape[0], 1) + 2) for x in la]
    gB = [_guarded(x, max(x.shape[0], 1) + 1) for x in lb]
    gC = [_guarded(x, max(x.shape[0], 1) + 3) for x in lc]
    ld = lambda xs, g: [max(x.shape[0], 1) + g for x in xs]
    h.summa(p, q, b, b, b, M, N, K, 1.5, [g[1] for g in gA], ld(la, 2), [g[1] for g in gB], ld(lb, 1), -0.5,
            [g[1] for g in gC], ld(lc, 3))
    torch.cuda.synchronize()
    h.check_device()
    for (t, _, img) in gA + gB:
        assert np.array_equal(t.cpu().numpy().view(np.uint64), img.view(np.uint64))
    res = []
    for x, (t, _, img) in zip(lc, gC):
        rows, cols = x.shape
        ldc = max(rows, 1) + 3
        got = t.cpu().numpy()
        inside = np.zeros(got.shape, dtype=bool)
        for j in range(cols):
            inside[GUARD + j * ldc:GUARD + j * ldc + rows] = True
        assert np.array_equal(got[~inside].view(np.uint64), img[~inside].view(np.uint64))
        res.append(np.stack([got[GUARD + j * ldc:GUARD + j * ldc + rows] for j in range(cols)], axis=1)
                   if rows and cols else np.zeros((rows, cols)))
    G = gather_block_cyclic(res, M, N, b, b, p, q)
    assert O.rel_errors(G, O.dgemm(A, B, 1.5, -0.5, C))[1] <= 1e-13


def test_nccl_driver_one_rank_on_gpu(tmp_path):
    """pre_distributed_cannon25_nccl on a 1 x 1 x 1 grid (a one-rank gloo group, no collective
    runs): the multiply through DgtOps on the GPU, two runs, the gathered C and the log."""
    import datetime
    import socket

    import pandas as pd
    import torch.distributed as dist
    from dgt import csvlog
    from dgt.dist import pre_distributed_cannon25_nccl

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        C = pre_distributed_cannon25_nccl(1, 1, 256, 2, alpha=1.5, beta=-0.5, gather_results=True,
                                          log_dir=str(tmp_path), machine="b200test", seed=5)
    finally:
        dist.destroy_process_group()
    rng = np.random.Generator(np.random.PCG64(5))
    A, B, C0 = (rng.uniform(-1.0, 1.0, (256, 256)) for _ in range(3))
    AB = A @ B
    want = 1.5 * AB - 0.5 * (1.5 * AB - 0.5 * C0)
    assert O.rel_errors(C, want)[1] <= 1e-13
    df = pd.read_csv(tmp_path / csvlog.cannon_nccl_log_name("b200test"), header=0)
    assert len(df) == 2 and (df["GFlops"] > 0).all()
