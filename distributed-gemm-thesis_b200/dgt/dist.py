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
