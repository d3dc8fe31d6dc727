"""SUMMA across processes: one process per GPU, the p x q process grid made physical.

The in-device schedule (dgt_summa) runs every virtual rank of the grid on one GPU, where
a panel broadcast is a panel read.  Here each rank is a process with its own device, and
the panels move between devices as torch.distributed broadcasts (NCCL over NVLink on
B200) on the process row and column sub-groups -- the physical step loop of the
reference's NCCL variant (src/25DCannonNCCL.cpp:109-304) applied to the block-cyclic
SUMMA whose contract is the cuBLASMp path (src/Wrappers/cuBLASMp/cuBLASMpValidator.cpp:45-50):

    for every K panel t (width kb, the last one ragged):
        process column t mod q broadcasts its local A block column t div q along each row,
        process row    t mod p broadcasts its local B block row    t div p along each column,
        every rank:    C_loc = alpha A_panel B_panel + (beta if t == 0 else 1) C_loc

Layout (the same as dgt_summa's): A is M x K in (mb x kb) blocks, B is K x N in (kb x nb)
blocks, C is M x N in (mb x nb) blocks, block-cyclic over the grid, rank r = i q + j.  Each
rank passes its local blocks as torch tensors of shape (local columns, local rows): the
column-major local matrix with leading dimension = local rows (numroc), the layout
dgt_pack_block_cyclic produces with dense locals.

Step t + 1's broadcasts are issued before step t's GEMM (one panel of lookahead, double
buffered), so on NCCL the transfer overlaps the multiply.  This is the collective-library
form of the step loop; the local GEMM and the panel packing are the library's kernels
(dgt_dgemm, dgt_copy_block) through `DgtOps`.  Tests substitute a host double for the
ops to run the same schedule as gloo ranks on the CPU.
"""
from __future__ import annotations

import math
import os

import dgt


def local_rows(n: int, nb: int, iproc: int, nprocs: int) -> int:
    return dgt.numroc(n, nb, iproc, 0, nprocs)


class DgtOps:
    """Local operations of a rank on its device, through the C ABI (the product path)."""

    def __init__(self, handle: "dgt.Handle", mode: int = dgt.FP64_NATIVE, slices: int = 7):
        self.h, self.mode, self.slices = handle, mode, slices

    def empty(self, shape, like):
        import torch

        return torch.empty(shape, dtype=torch.float64, device=like.device)

    def pack_rows(self, src, r0, rows, dst):
        """dst (cols x rows) <- rows r0 .. r0+rows of the column-major matrix src (cols x ld)."""
        cols, ld = src.shape
        self.h.copy_block(rows, cols, src.data_ptr() + 8 * r0, dst.data_ptr(), ld, rows)

    def copy(self, src, dst):
        """dst <- src for two contiguous tensors of the same shape (one strided-copy launch)."""
        cols, rows = src.shape
        self.h.copy_block(rows, cols, src.data_ptr(), dst.data_ptr(), rows, rows)

    def gemm(self, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
        """C = alpha A B + beta C on column-major device buffers (tensors' storage)."""
        self.h.dgemm("N", "N", m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta, C.data_ptr(), ldc,
                     mode=self.mode, slices=self.slices)


class DistSumma:
    """SUMMA on a p x q grid of processes (torch.distributed world of p*q ranks)."""

    def __init__(self, p: int, q: int, mb: int, nb: int, kb: int, ops=None):
        import torch.distributed as dist

        if not dist.is_initialized():
            raise RuntimeError("DistSumma needs an initialised torch.distributed process group")
        if min(p, q, mb, nb, kb) <= 0:
            raise ValueError("grid and block sizes must be positive")
        world, rank = dist.get_world_size(), dist.get_rank()
        if world != p * q:
            raise ValueError(f"world size {world} != p*q = {p * q}")
        self.p, self.q, self.mb, self.nb, self.kb = p, q, mb, nb, kb
        self.rank, self.i, self.j = rank, rank // q, rank % q
        # every rank creates every sub-group, in the same order
        self.row_groups = [dist.new_group([i * q + j for j in range(q)]) if q > 1 else None for i in range(p)]
        self.col_groups = [dist.new_group([i * q + j for i in range(p)]) if p > 1 else None for j in range(q)]
        self.ops = ops

    def local_shapes(self, M: int, N: int, K: int):
        """(rows, cols) of this rank's local A, B and C."""
        p, q, i, j = self.p, self.q, self.i, self.j
        return ((local_rows(M, self.mb, i, p), local_rows(K, self.kb, j, q)),
                (local_rows(K, self.kb, i, p), local_rows(N, self.nb, j, q)),
                (local_rows(M, self.mb, i, p), local_rows(N, self.nb, j, q)))

    def multiply(self, M: int, N: int, K: int, alpha: float, A_loc, B_loc, beta: float, C_loc) -> None:
        """C = alpha A B + beta C on the block-cyclic local tensors (in place in C_loc)."""
        import torch.distributed as dist

        if self.ops is None:
            import torch

            # the library works on torch's current stream, which NCCL's streams order against
            self.ops = DgtOps(dgt.Handle(stream=torch.cuda.current_stream().cuda_stream))
        ops = self.ops
        (ma, ka), (kb_rows, nbc), (m, n) = self.local_shapes(M, N, K)
        for name, t, rows, cols in (("A", A_loc, ma, ka), ("B", B_loc, kb_rows, nbc), ("C", C_loc, m, n)):
            if tuple(t.shape) != (max(cols, 1), max(rows, 1)) and not (rows == 0 or cols == 0):
                raise ValueError(f"local {name} must have shape (cols, rows) = ({cols}, {rows}), got {tuple(t.shape)}")
        p, q, i, j, kb = self.p, self.q, self.i, self.j, self.kb
        T = math.ceil(K / kb) if K > 0 else 0
        row_g, col_g = self.row_groups[i], self.col_groups[j]
        bufA = [None, None]
        bufB = [None, None]
        pending = {}

        def issue(t):
            kt = min(kb, K - t * kb)
            works = []
            # A panel t: process column t mod q, local columns (t div q) kb .. + kt.  Every
            # rank of process row i has the same ma, so a row skips (or joins) as a whole;
            # a rank without C columns still joins its row's and column's broadcasts.
            ra = t % q
            if ma > 0:
                if j == ra:
                    c0 = (t // q) * kb
                    a = A_loc[c0:c0 + kt]  # contiguous (kt, m) view: full local columns
                else:
                    if bufA[t % 2] is None or tuple(bufA[t % 2].shape) != (kt, ma):
                        bufA[t % 2] = ops.empty((kt, ma), C_loc)
                    a = bufA[t % 2]
                if row_g is not None:
                    works.append(dist.broadcast(a, src=i * q + ra, group=row_g, async_op=True))
            else:
                a = None
            # B panel t: process row t mod p, local rows (t div p) kb .. + kt
            rb = t % p
            if nbc > 0:
                if bufB[t % 2] is None or tuple(bufB[t % 2].shape) != (nbc, kt):
                    bufB[t % 2] = ops.empty((nbc, kt), C_loc)
                b = bufB[t % 2]
                if i == rb:
                    ops.pack_rows(B_loc, (t // p) * kb, kt, b)
                if col_g is not None:
                    works.append(dist.broadcast(b, src=rb * q + j, group=col_g, async_op=True))
            else:
                b = None
            pending[t] = (kt, a, b, works)

        if T == 0:
            if m > 0 and n > 0:
                ops.gemm(m, n, 0, alpha, C_loc, m, C_loc, 1, beta, C_loc, C_loc.shape[1])
            return
        issue(0)
        for t in range(T):
            if t + 1 < T:
                issue(t + 1)
            kt, a, b, works = pending.pop(t)
            for w in works:
                w.wait()
            if m > 0 and n > 0:
                ops.gemm(m, n, kt, alpha, a, m, b, kt, beta if t == 0 else 1.0, C_loc, C_loc.shape[1])


class DistCannon25D:
    """2.5D Cannon on a p x p x c grid of processes (world of p*p*c ranks), the reference's
    NCCL variant (Summa25Decomposer::multiplyNCCL, src/25DCannonNCCL.cpp:109-304) with the
    tiles of square M = N = K split in (M/p)^2 blocks:

      rank r = k p^2 + i p + j  (src/25DCannon.cpp:37-42)
      1. stack broadcast: stack 0's A_ij, B_ij to every stack (broadcastToStackNCCL, :84-96)
      2. skew: A_ij to column (j - i + k pc3) mod p, B_ij to row (i - j + k pc3) mod p (:120-126)
      3. pc3 = p / c steps: C += A B, then A moves one column right and B one row down
      4. stack reduce: C_ij(0) = sum over stacks (reduceResultNCCL, :306-320)

    so rank (i, j, k) multiplies k-blocks (i + j - k pc3 - r) mod p, r = 0 .. pc3 - 1, and the
    stacks together visit every k-block once.  The reference rotates by a growing amount
    (column j + r at step r), which skips k-blocks on some grids (p = 3, c = 1); unit shifts
    are the standard Cannon order and cover every grid.  Beta scales C on stack 0's first
    step; the other stacks start their partial sums from zero.  The caller's A and B tiles
    are read, never shifted in place (the reference's are, so its next call starts skewed).
    Each rank passes (M/p, M/p) tensors: column-major tiles with ld = M/p; after the call
    stack 0's C tiles hold the result.  Step r + 1's shifts are posted before step r's GEMM.
    """

    def __init__(self, p: int, c: int, ops=None):
        import torch.distributed as dist

        if not dist.is_initialized():
            raise RuntimeError("DistCannon25D needs an initialised torch.distributed process group")
        if p <= 0 or c <= 0 or p % c:
            raise ValueError("need p >= 1, c >= 1 and p % c == 0")
        world, rank = dist.get_world_size(), dist.get_rank()
        if world != p * p * c:
            raise ValueError(f"world size {world} != p*p*c = {p * p * c}")
        self.p, self.c, self.pc3 = p, c, p // c
        self.rank = rank
        self.k, self.i, self.j = rank // (p * p), (rank // p) % p, rank % p
        # every rank creates every stack fiber group, in the same order
        self.fibers = ([dist.new_group([k * p * p + r for k in range(c)]) for r in range(p * p)] if c > 1 else None)
        self.ops = ops

    def _rank_of(self, i, j, k=None):
        p = self.p
        return (self.k if k is None else k) * p * p + (i % p) * p + (j % p)

    def multiply(self, M: int, alpha: float, A_tile, B_tile, beta: float, C_tile) -> None:
        import torch.distributed as dist

        if self.ops is None:
            import torch

            self.ops = DgtOps(dgt.Handle(stream=torch.cuda.current_stream().cuda_stream))
        ops, p, c, pc3, i, j, k = self.ops, self.p, self.c, self.pc3, self.i, self.j, self.k
        if M <= 0 or M % p:
            raise ValueError("need M > 0 and M % p == 0")
        lm = M // p
        for name, t in (("A", A_tile), ("B", B_tile), ("C", C_tile)):
            if tuple(t.shape) != (lm, lm):
                raise ValueError(f"{name} tile must have shape ({lm}, {lm}), got {tuple(t.shape)}")

        # 1. stack broadcast of A and B (stack 0 sends its own tiles)
        if c > 1:
            fiber = self.fibers[i * p + j]
            root = self._rank_of(i, j, 0)
            if k == 0:
                a0, b0 = A_tile, B_tile
            else:
                a0, b0 = ops.empty((lm, lm), C_tile), ops.empty((lm, lm), C_tile)
            works = [dist.broadcast(a0, src=root, group=fiber, async_op=True),
                     dist.broadcast(b0, src=root, group=fiber, async_op=True)]
            for w in works:
                w.wait()
        else:
            a0, b0 = A_tile, B_tile

        ws_a = [ops.empty((lm, lm), C_tile), ops.empty((lm, lm), C_tile)] if p > 1 else None
        ws_b = [ops.empty((lm, lm), C_tile), ops.empty((lm, lm), C_tile)] if p > 1 else None

        def exchange(send_a, to_a, recv_a, from_a, send_b, to_b, recv_b, from_b):
            """Post the A and B moves of one shift; a move to oneself is a local copy."""
            ops_list = []
            for snd, to, rcv, frm in ((send_a, to_a, recv_a, from_a), (send_b, to_b, recv_b, from_b)):
                if to == self.rank and frm == self.rank:
                    ops.copy(snd, rcv)
                    continue
                ops_list.append(dist.P2POp(dist.isend, snd, to))
                ops_list.append(dist.P2POp(dist.irecv, rcv, frm))
            return dist.batch_isend_irecv(ops_list) if ops_list else []

        # 2. skew (reference convention); a tile that stays put is used in place
        kp = k * pc3
        if p > 1:
            reqs = exchange(a0, self._rank_of(i, j - i + kp), ws_a[0], self._rank_of(i, j + i - kp),
                            b0, self._rank_of(i - j + kp, j), ws_b[0], self._rank_of(i + j - kp, j))
            for r in reqs:
                r.wait()
            cur_a, cur_b = ws_a[0], ws_b[0]
        else:
            cur_a, cur_b = a0, b0

        # 3. steps, the next shift posted before this step's GEMM
        for r in range(pc3):
            reqs = []
            if r + 1 < pc3:
                nxt_a, nxt_b = ws_a[(r + 1) % 2], ws_b[(r + 1) % 2]
                reqs = exchange(cur_a, self._rank_of(i, j + 1), nxt_a, self._rank_of(i, j - 1),
                                cur_b, self._rank_of(i + 1, j), nxt_b, self._rank_of(i - 1, j))
            step_beta = (beta if k == 0 else 0.0) if r == 0 else 1.0
            ops.gemm(lm, lm, lm, alpha, cur_a, lm, cur_b, lm, step_beta, C_tile, lm)
            for q_ in reqs:
                q_.wait()
            if r + 1 < pc3:
                cur_a, cur_b = nxt_a, nxt_b

        # 4. stack reduction into stack 0
        if c > 1:
            dist.reduce(C_tile, dst=self._rank_of(i, j, 0), op=dist.ReduceOp.SUM, group=self.fibers[i * p + j])


class DeviceIpc:
    """Device buffers shared between the processes of a node through the C ABI's CUDA IPC
    entry points (dgt_ipc_*): a mapped peer buffer is read over NVLink by the kernels."""

    def __init__(self):
        self.lib = dgt.load()

    def alloc(self, nbytes: int):
        import ctypes

        ptr, h = ctypes.c_void_p(), ctypes.create_string_buffer(64)
        st = self.lib.dgt_ipc_alloc(max(int(nbytes), 8), ctypes.byref(ptr), h)
        if st != dgt.SUCCESS:
            raise dgt.DgtError(st, "dgt_ipc_alloc")
        return ptr.value, h.raw

    def open(self, handle: bytes) -> int:
        import ctypes

        ptr = ctypes.c_void_p()
        st = self.lib.dgt_ipc_open(ctypes.create_string_buffer(handle, 64), ctypes.byref(ptr))
        if st != dgt.SUCCESS:
            raise dgt.DgtError(st, "dgt_ipc_open")
        return ptr.value

    def close(self, ptr: int) -> None:
        self.lib.dgt_ipc_close(ptr)

    def free(self, ptr: int) -> None:
        self.lib.dgt_ipc_free(ptr)

    def tensor(self, ptr: int, shape):
        """A float64 torch tensor over device memory at ptr (no copy)."""
        import torch

        class _Buf:
            __cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                        "strides": None}

        return torch.as_tensor(_Buf(), device="cuda")

    def synchronize(self) -> None:
        import torch

        torch.cuda.synchronize()


class PeerSumma:
    """SUMMA across processes with the panel broadcasts fused into the GEMM: every rank's
    local A and B live in buffers the other ranks map (DeviceIpc), and each rank's
    dgt_summa_rank reads the owners' panels straight from their memory, tile by tile, as it
    multiplies -- no broadcast, no staging copy.  Same layout and result as DistSumma.

        S = PeerSumma(p, q, mb, nb, kb, M, N, K)      # collective: allocates and maps
        S.A_loc[...] = ...; S.B_loc[...] = ...          # this rank's block-cyclic locals
        S.multiply(alpha, beta, C_loc)                  # C_loc: (n, m) tensor, column-major
        S.close()                                       # collective

    Host barriers bracket each multiply (every owner's A and B are written before any rank
    reads them, and no owner rewrites them while a peer still reads); no kernel waits on
    another process.
    """

    def __init__(self, p, q, mb, nb, kb, M, N, K, ipc=None, handle=None, mode=dgt.FP64_NATIVE, slices=7):
        import torch.distributed as dist

        if not dist.is_initialized():
            raise RuntimeError("PeerSumma needs an initialised torch.distributed process group")
        if min(p, q, mb, nb, kb) <= 0 or min(M, N, K) < 0:
            raise ValueError("grid, block sizes and dimensions must be valid")
        world, rank = dist.get_world_size(), dist.get_rank()
        if world != p * q:
            raise ValueError(f"world size {world} != p*q = {p * q}")
        self.p, self.q, self.mb, self.nb, self.kb, self.M, self.N, self.K = p, q, mb, nb, kb, M, N, K
        self.rank, self.mode, self.slices = rank, mode, slices
        self.ipc = ipc or DeviceIpc()
        if handle is None:
            import torch

            handle = dgt.Handle(stream=torch.cuda.current_stream().cuda_stream)
        self.h = handle
        P = p * q
        self.lldA = [max(1, local_rows(M, mb, r // q, p)) for r in range(P)]
        self.lldB = [max(1, local_rows(K, kb, r // q, p)) for r in range(P)]
        colsA = max(1, local_rows(K, kb, rank % q, q))
        colsB = max(1, local_rows(N, nb, rank % q, q))
        self._own, opened = [], []
        try:
            self._own.append(self.ipc.alloc(8 * self.lldA[rank] * colsA))
            self._own.append(self.ipc.alloc(8 * self.lldB[rank] * colsB))
            handles = [None] * world
            dist.all_gather_object(handles, (self._own[0][1], self._own[1][1]))
            self.A_ptrs, self.B_ptrs = [], []
            for r in range(P):
                for ptrs, own, h in ((self.A_ptrs, self._own[0][0], handles[r][0]),
                                     (self.B_ptrs, self._own[1][0], handles[r][1])):
                    if r == rank:
                        ptrs.append(own)
                    else:
                        ptrs.append(self.ipc.open(h))
                        opened.append(ptrs[-1])
        except Exception:
            # give back what this rank took; peers see the failure at their next collective
            for ptr in opened:
                self.ipc.close(ptr)
            for ptr, _ in self._own:
                self.ipc.free(ptr)
            self._own = []
            raise
        self.A_loc = self.ipc.tensor(self._own[0][0], (colsA, self.lldA[rank]))
        self.B_loc = self.ipc.tensor(self._own[1][0], (colsB, self.lldB[rank]))
        self.m = local_rows(M, mb, rank // q, p)
        self.n = local_rows(N, nb, rank % q, q)

    def multiply(self, alpha: float, beta: float, C_loc) -> None:
        import torch.distributed as dist

        if tuple(C_loc.shape) != (max(self.n, 1), max(self.m, 1)):
            raise ValueError(f"C_loc must have shape ({max(self.n, 1)}, {max(self.m, 1)})")
        self.ipc.synchronize()
        dist.barrier()
        self.h.summa_rank(self.rank, self.p, self.q, self.mb, self.nb, self.kb, self.M, self.N, self.K, alpha,
                          self.A_ptrs, self.lldA, self.B_ptrs, self.lldB, beta, C_loc.data_ptr(), max(self.m, 1),
                          mode=self.mode, slices=self.slices)
        self.ipc.synchronize()
        dist.barrier()

    def close(self) -> None:
        import torch.distributed as dist

        for r, (a, b) in enumerate(zip(self.A_ptrs, self.B_ptrs)):
            if r != self.rank:
                self.ipc.close(a)
                self.ipc.close(b)
        dist.barrier()
        for ptr, _ in self._own:
            self.ipc.free(ptr)
        self._own = []


class PeerCannon25D:
    """2.5D Cannon across p*p*c processes with its communication fused into the kernels: the
    stack-0 ranks hold A_ij and B_ij in buffers every rank maps (DeviceIpc), each rank's
    dgt_cannon25d_rank reads the tiles of its k-blocks straight from their owners (no stack
    broadcast, no skew, no shifts), and each stack-0 rank sums the other stacks' partials
    by reading them from their ranks (dgt_reduce_tiles) -- the reduction reads the partial
    sums where the GEMMs left them.  Same k-block order and summation order as the in-device
    dgt_cannon25d.

        S = PeerCannon25D(p, c, M)            # collective
        S.A_tile[...] = ...; S.B_tile[...] = ...  (stack-0 ranks: tile (i, j), column-major)
        S.multiply(alpha, beta, C_tile)       # stack 0: the C tile, result in place
        S.close()                             # collective

    Host barriers separate publishing the tiles, the GEMMs, and the reduction; no kernel
    waits on another process.
    """

    def __init__(self, p, c, M, ipc=None, handle=None, mode=dgt.FP64_NATIVE, slices=7):
        import torch.distributed as dist

        if not dist.is_initialized():
            raise RuntimeError("PeerCannon25D needs an initialised torch.distributed process group")
        if p <= 0 or c <= 0 or p % c or M <= 0 or M % p:
            raise ValueError("need p % c == 0 and M % p == 0")
        world, rank = dist.get_world_size(), dist.get_rank()
        if world != p * p * c:
            raise ValueError(f"world size {world} != p*p*c = {p * p * c}")
        self.p, self.c, self.M, self.lm, self.rank = p, c, M, M // p, rank
        self.k, self.i, self.j = rank // (p * p), (rank // p) % p, rank % p
        self.mode, self.slices = mode, slices
        self.ipc = ipc or DeviceIpc()
        if handle is None:
            import torch

            handle = dgt.Handle(stream=torch.cuda.current_stream().cuda_stream)
        self.h = handle
        nbytes = 8 * self.lm * self.lm
        self._own, opened = [], []
        try:
            # stack 0 owns the A and B tiles; the other stacks own their partial C
            names = ("A", "B") if self.k == 0 else ("P",)
            mine = {}
            for name in names:
                ptr, hnd = self.ipc.alloc(nbytes)
                self._own.append((ptr, hnd))
                mine[name] = (ptr, hnd)
            handles = [None] * world
            dist.all_gather_object(handles, {n: h for n, (_, h) in mine.items()})

            def mapped(r, name):
                if r == rank:
                    return mine[name][0]
                ptr = self.ipc.open(handles[r][name])
                opened.append(ptr)
                return ptr

            self.A_ptrs = [mapped(r, "A") for r in range(p * p)]
            self.B_ptrs = [mapped(r, "B") for r in range(p * p)]
            base = self.i * p + self.j
            self.P_ptrs = [mapped(k * p * p + base, "P") for k in range(1, c)] if self.k == 0 else []
        except Exception:
            for ptr in opened:
                self.ipc.close(ptr)
            for ptr, _ in self._own:
                self.ipc.free(ptr)
            self._own = []
            raise
        self._opened = opened
        self.A_tile = self.ipc.tensor(mine["A"][0], (self.lm, self.lm)) if self.k == 0 else None
        self.B_tile = self.ipc.tensor(mine["B"][0], (self.lm, self.lm)) if self.k == 0 else None
        self._partial = mine["P"][0] if self.k > 0 else None

    def multiply(self, alpha: float, beta: float, C_tile=None) -> None:
        import torch.distributed as dist

        if self.k == 0 and (C_tile is None or tuple(C_tile.shape) != (self.lm, self.lm)):
            raise ValueError(f"stack-0 ranks pass their ({self.lm}, {self.lm}) C tile")
        c_ptr = C_tile.data_ptr() if self.k == 0 else self._partial
        self.ipc.synchronize()
        dist.barrier()  # every stack-0 tile is published
        self.h.cannon25d_rank(self.M, self.p, self.c, self.rank, alpha, self.A_ptrs, self.B_ptrs, beta, c_ptr,
                              mode=self.mode, slices=self.slices)
        self.ipc.synchronize()
        dist.barrier()  # every partial is complete
        if self.k == 0 and self.P_ptrs:
            self.h.reduce_tiles(c_ptr, self.P_ptrs, self.lm * self.lm)
            self.ipc.synchronize()
        dist.barrier()  # no partial or tile is read any more

    def close(self) -> None:
        import torch.distributed as dist

        for ptr in self._opened:
            self.ipc.close(ptr)
        self._opened = []
        dist.barrier()
        for ptr, _ in self._own:
            self.ipc.free(ptr)
        self._own = []


def pre_distributed_cannon25_nccl(p, c, M, runs, alpha=1.0, beta=0.0, logging=True, gather_results=False,
                                  log_dir=".", machine=None, fused=False, seed=0, ops=None, ipc=None, handle=None,
                                  sync=None):
    """The reference's NCCL benchmark driver (preDistributedCannon25NCCL,
    src/25DCannonNCCL.cpp:322-399) over the multi-process 2.5D Cannon: one process per GPU,
    p*p*c ranks.  DecompositionTime is the decomposer's construction, as in the reference
    (:343-345); the stack-0 tiles are then filled with U[-1, 1) values (global A, B, C from
    numpy's PCG64(seed), tile (i, j) of each); every run is one multiply, timed between two
    barriers (the slowest rank's time); with gather_results the stack-0 C tiles are
    collected on rank 0 (reorderMatrix).  Rank 0 appends one row per run in the reference's
    NCCL schema (Algo "2.5D CANNON dgt NCCL", or "2.5D CANNON dgt peer" for the fused form;
    TotalGPUs = the number of ranks, one GPU each).  Returns C on rank 0 when gathering,
    else None.  `fused` selects PeerCannon25D (kernels read the owners' tiles) instead of
    DistCannon25D (NCCL broadcasts and shifts); ops / ipc / handle / sync stand in for the
    device in tests."""
    import time

    import numpy as np
    import torch
    import torch.distributed as dist

    from . import csvlog

    rank, world = dist.get_rank(), dist.get_world_size()
    if sync is None:
        sync = torch.cuda.synchronize
    log = None
    if logging and rank == 0:
        name = csvlog.cannon_nccl_log_name(machine or csvlog.machine_name())
        log = csvlog.create_log_csv(os.path.join(log_dir, name), csvlog.CANNON_NCCL_HEADER)
    try:
        t0 = time.perf_counter()
        S = (PeerCannon25D(p, c, M, ipc=ipc, handle=handle) if fused else DistCannon25D(p, c, ops=ops))
        decomp = time.perf_counter() - t0
        lm = M // p
        k, i, j = rank // (p * p), (rank // p) % p, rank % p
        device = "cpu" if (ops is not None or ipc is not None) else "cuda"
        rng = np.random.Generator(np.random.PCG64(seed))
        G = [rng.uniform(-1.0, 1.0, (M, M)) for _ in range(3)]
        tile = lambda X: torch.from_numpy(np.ascontiguousarray(X[i * lm:(i + 1) * lm, j * lm:(j + 1) * lm].T)).to(device)
        if fused:
            C_tile = None
            if k == 0:
                S.A_tile.copy_(tile(G[0]))
                S.B_tile.copy_(tile(G[1]))
                C_tile = tile(G[2])
            A_tile = B_tile = None
        else:
            A_tile, B_tile = (tile(G[0]), tile(G[1])) if k == 0 else (torch.empty((lm, lm), dtype=torch.float64,
                                                                                   device=device),) * 2
            C_tile = tile(G[2]) if k == 0 else torch.empty((lm, lm), dtype=torch.float64, device=device)
        result = None
        for _ in range(runs):
            sync()
            dist.barrier()
            t0 = time.perf_counter()
            if fused:
                S.multiply(alpha, beta, C_tile)
            else:
                S.multiply(M, alpha, A_tile, B_tile, beta, C_tile)
            sync()
            dist.barrier()
            execution = time.perf_counter() - t0
            t0 = time.perf_counter()
            if gather_results:
                mine = C_tile.cpu().numpy().T.copy() if k == 0 else None
                tiles = [None] * world if rank == 0 else None
                dist.gather_object(mine, tiles, dst=0)
                if rank == 0:
                    result = np.zeros((M, M))
                    for r in range(p * p):
                        ri, rj = r // p, r % p
                        result[ri * lm:(ri + 1) * lm, rj * lm:(rj + 1) * lm] = tiles[r]
            gather = time.perf_counter() - t0
            if log is not None:
                algo = "2.5D CANNON dgt peer" if fused else "2.5D CANNON dgt NCCL"
                csvlog.write_line_to_file(log, csvlog.cannon_nccl_row(
                    algo, M, M, M, csvlog.slurm_num_nodes(), world, p, p, c, decomp, execution, gather,
                    csvlog.calculate_gflops(M, M, M, execution)))
        if fused:
            S.close()
        return result
    finally:
        if log is not None:
            log.close()


# ---- benchmark of the physical step loop --------------------------------------------------------

class DeviceClock:
    """Device time of a region on torch's current stream (the stream the library's kernels
    and, ordered against it, NCCL's run on): CUDA events, synchronized on both sides."""

    def start(self) -> None:
        import torch

        torch.cuda.synchronize()
        self.e0, self.e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        self.e0.record()

    def stop(self) -> float:
        import torch

        self.e1.record()
        torch.cuda.synchronize()
        return self.e0.elapsed_time(self.e1)


class HostClock:
    """Wall time of a region (the host doubles' clock)."""

    def start(self) -> None:
        import time

        self.t0 = time.perf_counter()

    def stop(self) -> float:
        import time

        return (time.perf_counter() - self.t0) * 1e3


def _max_over_ranks(x: float) -> float:
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def summa_benchmark(M: int, N: int, K: int, mb: int, nb: int, kb: int, steps: int = 3, warmup: int = 1,
                    alpha: float = 1.0, beta: float = 0.0, ops=None, ipc=None, handle=None, clock=None,
                    device: str = "cuda", seed: int = 0) -> dict:
    """Times the physical SUMMA step loop on this process group: the world's p x q grid is the
    reference's most-square factorisation (calculateVirtualDeviceGrid,
    src/Decompositions/2DBlockSequentialDecomposition.cpp:27-54), every rank fills its
    block-cyclic locals of A, B and C from its own seeded generator, and two forms run the
    same product:

      * collective -- DistSumma: panels broadcast on the process-row / -column sub-groups
        (NCCL on B200), one panel of lookahead, the local GEMMs through the C ABI;
      * fused      -- PeerSumma: every rank's dgt_summa_rank reads the owners' panels from
        their memory (CUDA IPC, plain loads), no broadcast.

    Each form: `warmup` untimed multiplies, then `steps` timed ones between barriers; the time
    is the maximum over ranks.  The compute reference is the same rank's m x n x K product as
    one local GEMM with no communication (dense local operands), so exposed communication =
    form time - compute time.  Returns a dict with, per form, ms per multiply, whole-job
    TFLOP/s (2 M N K / time), the compute reference and the exposed communication, plus the
    fused result's relative Frobenius distance from the collective one on this rank (max over
    ranks; the two differ only in summation order).  `ops`, `ipc`, `handle` and `clock` take
    the host doubles on CPU; on a GPU they default to the library (DgtOps, DeviceIpc,
    dgt.Handle on torch's current stream) and CUDA events."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size()
    rank = dist.get_rank()
    p, q = dgt.block2d_grid(world)
    clock = clock or DeviceClock()
    own_handle = device == "cuda" and handle is None
    if own_handle:
        handle = dgt.Handle(stream=torch.cuda.current_stream().cuda_stream)
    try:
        return _summa_benchmark(M, N, K, mb, nb, kb, steps, warmup, alpha, beta, ops or DgtOps(handle), ipc, handle,
                                clock, device, seed, world, rank, p, q)
    finally:
        if own_handle:
            handle.close()


def _summa_benchmark(M, N, K, mb, nb, kb, steps, warmup, alpha, beta, ops, ipc, handle, clock, device, seed, world,
                     rank, p, q):
    import torch
    import torch.distributed as dist

    gen = torch.Generator(device=device)
    gen.manual_seed(seed * 1000 + rank)

    def rand(shape):
        return torch.rand(shape, dtype=torch.float64, device=device, generator=gen) * 2 - 1

    def timed(fn) -> float:
        for _ in range(warmup):
            fn()
        dist.barrier()
        clock.start()
        for _ in range(steps):
            fn()
        ms = clock.stop() / max(steps, 1)
        dist.barrier()
        return _max_over_ranks(ms)

    S = DistSumma(p, q, mb, nb, kb, ops=ops)
    (ma, ka), (kr, nc), (m, n) = S.local_shapes(M, N, K)
    A_loc, B_loc = rand((max(ka, 1), max(ma, 1))), rand((max(nc, 1), max(kr, 1)))
    C0 = rand((max(n, 1), max(m, 1)))
    C_coll = C0.clone()
    # both forms run warmup + steps multiplies from the same C0, so their results compare
    coll_ms = timed(lambda: S.multiply(M, N, K, alpha, A_loc, B_loc, beta, C_coll))

    # compute reference: this rank's m x n x K as one local GEMM on dense local operands
    if m > 0 and n > 0 and K > 0:
        A_full, B_full, C_full = rand((K, m)), rand((n, K)), C0.clone()
        comp_ms = timed(lambda: ops.gemm(m, n, K, alpha, A_full, m, B_full, K, beta, C_full, m))
        del A_full, B_full, C_full
    else:
        comp_ms = timed(lambda: None)

    P = PeerSumma(p, q, mb, nb, kb, M, N, K, ipc=ipc, handle=handle)
    try:
        P.A_loc.copy_(A_loc)
        P.B_loc.copy_(B_loc)
        C_fused = C0.clone()
        fused_ms = timed(lambda: P.multiply(alpha, beta, C_fused))
        if device == "cuda":
            torch.cuda.synchronize()
        den = float(torch.linalg.norm(C_coll)) or 1.0
        diff = _max_over_ranks(float(torch.linalg.norm(C_fused - C_coll)) / den)
    finally:
        P.close()
    flops = 2.0 * M * N * K

    def form(ms):
        return {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12 if ms > 0 else 0.0, "compute_ms": comp_ms,
                "exposed_comm_ms": max(ms - comp_ms, 0.0)}

    return {"grid": [p, q], "M": M, "N": N, "K": K, "blocks": [mb, nb, kb], "ranks": world,
            "collective": form(coll_ms), "fused": form(fused_ms), "fused_vs_collective_rel": diff}
