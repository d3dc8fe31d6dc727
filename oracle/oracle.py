"""ORACLE -- test infrastructure only.

CPU checker for the dgemm-b200 hot path.  Three parts:

* ``orc``: ctypes view of ``liborc.so`` (orc.c), the C restatement of the reference's
  layout routines and Cannon schedule (each C function cites the reference lines it
  follows), plus a double-double GEMM checker for sampled entries.
* ``ref``: ctypes view of ``_ref/libref.so`` -- the reference's OWN hot-path sources
  (src/Decompositions/*, src/Transfers/*, src/25DCannon.cpp) compiled by oracle/Makefile
  against in-process MPI / host-CUDA test doubles.  Present only where the reference
  tree was available at build time; tests fall back to the committed golden fixtures.
* numpy helpers: seeded input generators for every benchmark configuration and the
  FP64 GEMM oracle, which is host OpenBLAS ``dgemm`` (the reference validates with
  ``cblas_dgemm``: src/Wrappers/cuBLASMp/cuBLASMpValidator.cpp:48).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs may import this
module.  The product never does.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORC = os.path.join(HERE, "liborc.so")
_REF = os.path.join(HERE, "_ref", "libref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_ip = ctypes.POINTER(ctypes.c_int)


def build(ref_root: str | None = None) -> None:
    """Compile liborc.so and, when the reference tree exists, _ref/libref.so."""
    cmd = ["make", "-s", "-C", HERE, "all"]
    if ref_root:
        cmd.append(f"REF={ref_root}")
    subprocess.run(cmd, check=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _ptr_array(arrs):
    return (_dp * len(arrs))(*[_ptr(a) for a in arrs])


class _Orc:
    def __init__(self, path=_ORC):
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        self.L = L
        L.orc_numroc.restype = ctypes.c_int
        L.orc_numroc.argtypes = [ctypes.c_int] * 5
        L.orc_pblas_local_shape.argtypes = [ctypes.c_int] * 7 + [_ip, _ip, _ip]
        L.orc_pblas_scatter.argtypes = [ctypes.c_int] * 6 + [_dp, ctypes.c_int64, ctypes.c_void_p, _i64p]
        L.orc_pblas_scatter.restype = ctypes.c_int
        L.orc_pblas_gather.argtypes = [ctypes.c_int] * 6 + [_dp, ctypes.c_int64, ctypes.c_void_p, _i64p]
        L.orc_pblas_gather.restype = ctypes.c_int
        L.orc_block2d_grid.argtypes = [ctypes.c_int, _ip, _ip]
        L.orc_block2d_deliver.argtypes = [ctypes.c_int64] * 3 + [ctypes.c_int] * 3 + [_dp] * 3 + [ctypes.c_void_p] * 3
        L.orc_block2d_gather.argtypes = [ctypes.c_int64] * 2 + [ctypes.c_int] * 3 + [_dp, ctypes.c_void_p]
        L.orc_cannon_decompose.argtypes = [ctypes.c_int64, ctypes.c_int] + [_dp] * 3 + [ctypes.c_void_p] * 3
        L.orc_cannon_reorder.argtypes = [ctypes.c_int64, ctypes.c_int, _dp, ctypes.c_void_p]
        L.orc_cannon_schedule.argtypes = [ctypes.c_int] * 5 + [_ip]
        L.orc_cannon_schedule.restype = ctypes.c_int
        L.orc_copy_block.argtypes = [ctypes.c_int64] * 2 + [_dp, _dp] + [ctypes.c_int64] * 2 + [ctypes.c_int]
        L.orc_dgemm_dd_sample.argtypes = [ctypes.c_char, ctypes.c_char, ctypes.c_int64, ctypes.c_double, _dp,
                                          ctypes.c_int64, _dp, ctypes.c_int64, ctypes.c_double, _dp, ctypes.c_int64,
                                          ctypes.c_int64, _i64p, _i64p, _dp]
        L.orc_dd_rows.argtypes = [ctypes.c_int64, ctypes.c_int64, _dp, ctypes.c_int64, ctypes.c_int64, _dp,
                                  ctypes.c_int64, ctypes.c_double, _dp, ctypes.c_int64, ctypes.c_int]

    # -- block-cyclic --------------------------------------------------------------
    def numroc(self, n, nb, iproc, isrproc, nprocs):
        return self.L.orc_numroc(n, nb, iproc, isrproc, nprocs)

    def pblas_shapes(self, M, N, Mb, Nb, p, q):
        out = []
        for r in range(p * q):
            a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            self.L.orc_pblas_local_shape(M, N, Mb, Nb, p, q, r, a, b, c)
            out.append((a.value, b.value, c.value))
        return out

    def pblas_scatter(self, G, Mb, Nb, p, q):
        """Global column-major G -> list of local column-major arrays (ld = numroc rows)."""
        G = np.asfortranarray(G, dtype=np.float64)
        M, N = G.shape
        shapes = self.pblas_shapes(M, N, Mb, Nb, p, q)
        locs = [np.zeros((r, c), dtype=np.float64, order="F") for r, c, _ in shapes]
        lld = (ctypes.c_int64 * len(locs))(*[max(r, 1) for r, _, _ in shapes])
        rc = self.L.orc_pblas_scatter(M, N, Mb, Nb, p, q, _ptr(G), M, _ptr_array(locs), lld)
        if rc != 0:
            raise ValueError("block-cyclic grid leaves a rank without rows or columns")
        return locs

    def pblas_gather(self, locs, M, N, Mb, Nb, p, q):
        G = np.zeros((M, N), dtype=np.float64, order="F")
        locs = [np.asfortranarray(l) for l in locs]
        lld = (ctypes.c_int64 * len(locs))(*[max(l.shape[0], 1) for l in locs])
        rc = self.L.orc_pblas_gather(M, N, Mb, Nb, p, q, _ptr(G), M, _ptr_array(locs), lld)
        if rc != 0:
            raise ValueError("block-cyclic grid leaves a rank without rows or columns")
        return G

    # -- 2D block --------------------------------------------------------------------
    def block2d_grid(self, P):
        a, b = ctypes.c_int(), ctypes.c_int()
        self.L.orc_block2d_grid(P, a, b)
        return a.value, b.value

    @staticmethod
    def block2d_tiles(M, N, K, dRow, dCol):
        """(tileM, tileN) per rank, remainder on the last grid row/column."""
        out = []
        for i in range(dRow):
            for j in range(dCol):
                tm = M // dRow + (M % dRow if i + 1 == dRow else 0)
                tn = N // dCol + (N % dCol if j + 1 == dCol else 0)
                out.append((tm, tn))
        return out

    def block2d_deliver(self, A, B, C, P, col_major=True):
        M, K = A.shape
        N = B.shape[1]
        dRow, dCol = self.block2d_grid(P)
        order = "F" if col_major else "C"
        A = np.asarray(A, dtype=np.float64, order=order)
        B = np.asarray(B, dtype=np.float64, order=order)
        C = np.asarray(C, dtype=np.float64, order=order)
        tiles = self.block2d_tiles(M, N, K, dRow, dCol)
        lA = [np.zeros((tm, K), order=order) for tm, _ in tiles]
        lB = [np.zeros((K, tn), order=order) for _, tn in tiles]
        lC = [np.zeros((tm, tn), order=order) for tm, tn in tiles]
        self.L.orc_block2d_deliver(M, N, K, dRow, dCol, int(col_major), _ptr(A), _ptr(B), _ptr(C), _ptr_array(lA),
                                   _ptr_array(lB), _ptr_array(lC))
        return lA, lB, lC

    def block2d_gather(self, lC, M, N, P, col_major=True, C=None):
        dRow, dCol = self.block2d_grid(P)
        order = "F" if col_major else "C"
        C = np.zeros((M, N), order=order) if C is None else np.array(C, dtype=np.float64, order=order)
        lC = [np.asarray(l, dtype=np.float64, order=order) for l in lC]
        self.L.orc_block2d_gather(M, N, dRow, dCol, int(col_major), _ptr(C), _ptr_array(lC))
        return C

    # -- Cannon ----------------------------------------------------------------------
    def cannon_decompose(self, A, B, C, p):
        M = A.shape[0]
        A, B, C = (np.asfortranarray(x, dtype=np.float64) for x in (A, B, C))
        lm = M // p
        mk = lambda: [np.zeros((lm, lm), order="F") for _ in range(p * p)]
        lA, lB, lC = mk(), mk(), mk()
        self.L.orc_cannon_decompose(M, p, _ptr(A), _ptr(B), _ptr(C), _ptr_array(lA), _ptr_array(lB), _ptr_array(lC))
        return lA, lB, lC

    def cannon_reorder(self, lC, M, p, C=None):
        C = np.zeros((M, M), order="F") if C is None else np.array(C, dtype=np.float64, order="F")
        lC = [np.asfortranarray(l) for l in lC]
        self.L.orc_cannon_reorder(M, p, _ptr(C), _ptr_array(lC))
        return C

    def cannon_schedule(self, p, c, i, j, k):
        pc3 = int((p * p * c / c ** 3) ** 0.5 + 1e-9)
        out = (ctypes.c_int * max(pc3, 1))()
        ok = self.L.orc_cannon_schedule(p, c, i, j, k, out)
        return list(out)[:pc3], bool(ok)

    # -- extended-precision checker -----------------------------------------------------
    def dgemm_dd_sample(self, A, B, alpha, beta, C0, rows, cols, ta="N", tb="N"):
        A = np.asfortranarray(A, dtype=np.float64)
        B = np.asfortranarray(B, dtype=np.float64)
        K = A.shape[0] if ta.upper() != "N" else A.shape[1]
        C0p = _ptr(np.asfortranarray(C0)) if C0 is not None else None
        ldc = C0.shape[0] if C0 is not None else 1
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int64)
        out = np.zeros(len(rows))
        if C0 is not None:
            C0 = np.asfortranarray(C0)
            C0p = _ptr(C0)
        self.L.orc_dgemm_dd_sample(ta.encode(), tb.encode(), K, alpha, _ptr(A), A.shape[0], _ptr(B), B.shape[0],
                                   beta, C0p, ldc, len(rows), rows.ctypes.data_as(_i64p),
                                   cols.ctypes.data_as(_i64p), _ptr(out))
        return out


    def dd_rows(self, A_rows, B, alpha=1.0, threads=0):
        """alpha * A_rows @ B in double-double (TwoSum / TwoProduct), rounded once to double:
        the exact product of a few sampled rows (A_rows: r x K) with all of B (K x n), on
        `threads` host threads (0: every online core)."""
        At = np.ascontiguousarray(A_rows, dtype=np.float64)  # row s K-contiguous at At[s]
        B = np.asfortranarray(B, dtype=np.float64)
        r, K = At.shape
        n = B.shape[1]
        out = np.zeros((r, n), order="F")
        self.L.orc_dd_rows(K, r, _ptr(At), K, n, _ptr(B), B.shape[0], alpha, _ptr(out), r, int(threads))
        return out


class _Ref:
    """The reference's own code (oracle/_ref/libref.so)."""

    def __init__(self, path=_REF):
        L = ctypes.CDLL(path)
        self.L = L
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_numroc.argtypes = [ctypes.c_int] * 5
        L.ref_pblas_shapes.argtypes = [ctypes.c_int] * 6 + [_ip] * 3
        L.ref_pblas_scatter.argtypes = [ctypes.c_int] * 6 + [_dp, ctypes.c_void_p]
        L.ref_pblas_gather.argtypes = [ctypes.c_int] * 6 + [_dp, ctypes.c_void_p]
        L.ref_block2d_shapes.argtypes = [ctypes.c_int] * 4 + [_ip] * 4
        L.ref_block2d_deliver.argtypes = [ctypes.c_int] * 5 + [_dp] * 3 + [ctypes.c_void_p] * 3
        L.ref_block2d_gather.argtypes = [ctypes.c_int] * 6 + [_dp, ctypes.c_void_p]
        L.ref_cannon_decompose.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_int] + [_dp] * 3 + [
            ctypes.c_void_p] * 3
        L.ref_cannon_reorder.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_void_p]
        L.ref_cannon_fulloffload.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, _dp, _dp, _dp]
        L.ref_cannon_fulloffload_logged.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, ctypes.c_int]
        L.ref_cannon_trace.argtypes = [ctypes.c_int, ctypes.c_int, _ip]
        for name in ("ref_copy_block_f64", "ref_copy_block_f32"):
            getattr(L, name).argtypes = [ctypes.c_longlong] * 2 + [ctypes.c_void_p] * 2 + [ctypes.c_longlong] * 2 + [
                ctypes.c_int]
        L.ref_set_dgemm.argtypes = [ctypes.c_void_p]
        self._blas = None

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("reference run failed: " + self.L.ref_last_error().decode())

    def use_openblas(self, threads: int | None = None) -> bool:
        """Route the reference's cublasDgemm to host OpenBLAS (scipy's LP64 build)."""
        import scipy

        libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs",
                                      "libscipy_openblas-*.so"))
        if not libs:
            return False
        blas = ctypes.CDLL(libs[0])
        if threads:
            blas.scipy_openblas_set_num_threads(int(threads))
        self._blas = blas
        self.L.ref_set_dgemm(ctypes.cast(blas.scipy_cblas_dgemm, ctypes.c_void_p))
        return True

    def use_naive(self):
        self.L.ref_set_dgemm(None)

    def numroc(self, n, nb, iproc, isrproc, nprocs):
        return self.L.ref_numroc(n, nb, iproc, isrproc, nprocs)

    def pblas_shapes(self, M, N, Mb, Nb, p, q):
        P = p * q
        a, b, c = (ctypes.c_int * P)(), (ctypes.c_int * P)(), (ctypes.c_int * P)()
        self._check(self.L.ref_pblas_shapes(M, N, Mb, Nb, p, q, a, b, c))
        return [(a[r], b[r], c[r]) for r in range(P)]

    def pblas_scatter(self, G, Mb, Nb, p, q):
        G = np.asfortranarray(G, dtype=np.float64)
        M, N = G.shape
        shapes = self.pblas_shapes(M, N, Mb, Nb, p, q)
        locs = [np.zeros((r, c), order="F") for r, c, _ in shapes]
        self._check(self.L.ref_pblas_scatter(M, N, Mb, Nb, p, q, _ptr(G), _ptr_array(locs)))
        return locs

    def pblas_gather(self, locs, M, N, Mb, Nb, p, q):
        G = np.zeros((M, N), order="F")
        locs = [np.asfortranarray(l) for l in locs]
        self._check(self.L.ref_pblas_gather(M, N, Mb, Nb, p, q, _ptr(G), _ptr_array(locs)))
        return G

    def block2d_shapes(self, M, N, K, P):
        dr, dc = ctypes.c_int(), ctypes.c_int()
        lm, ln = (ctypes.c_int * P)(), (ctypes.c_int * P)()
        self._check(self.L.ref_block2d_shapes(M, N, K, P, dr, dc, lm, ln))
        return dr.value, dc.value, list(lm), list(ln)

    def block2d_deliver(self, A, B, C, P, col_major=True):
        M, K = A.shape
        N = B.shape[1]
        order = "F" if col_major else "C"
        A = np.asarray(A, dtype=np.float64, order=order)
        B = np.asarray(B, dtype=np.float64, order=order)
        C = np.asarray(C, dtype=np.float64, order=order)
        dr, dc, lm, ln = self.block2d_shapes(M, N, K, P)
        lA = [np.zeros((lm[r], K), order=order) for r in range(P)]
        lB = [np.zeros((K, ln[r]), order=order) for r in range(P)]
        lC = [np.zeros((lm[r], ln[r]), order=order) for r in range(P)]
        self._check(self.L.ref_block2d_deliver(M, N, K, P, int(col_major), _ptr(A), _ptr(B), _ptr(C),
                                               _ptr_array(lA), _ptr_array(lB), _ptr_array(lC)))
        return lA, lB, lC

    def block2d_gather(self, lC, M, N, K, P, col_major=True, C=None):
        order = "F" if col_major else "C"
        C = np.zeros((M, N), order=order) if C is None else np.array(C, dtype=np.float64, order=order)
        lC = [np.asarray(l, dtype=np.float64, order=order) for l in lC]
        self._check(self.L.ref_block2d_gather(M, N, K, P, int(col_major), 0, _ptr(C), _ptr_array(lC)))
        return C

    def cannon_decompose(self, A, B, C, p, c=1):
        M = A.shape[0]
        A, B, C = (np.array(x, dtype=np.float64, order="F") for x in (A, B, C))
        lm = M // p
        mk = lambda: [np.zeros((lm, lm), order="F") for _ in range(p * p * c)]
        lA, lB, lC = mk(), mk(), mk()
        self._check(self.L.ref_cannon_decompose(M, p, c, _ptr(A), _ptr(B), _ptr(C), _ptr_array(lA), _ptr_array(lB),
                                                _ptr_array(lC)))
        return lA[:p * p], lB[:p * p], lC[:p * p]

    def cannon_reorder(self, lC, M, p, c=1, C=None):
        C = np.zeros((M, M), order="F") if C is None else np.array(C, dtype=np.float64, order="F")
        lm = M // p
        tiles = [np.asfortranarray(l) for l in lC] + [np.zeros((lm, lm), order="F")] * (p * p * (c - 1))
        self._check(self.L.ref_cannon_reorder(M, p, c, _ptr(C), _ptr_array(tiles)))
        return C

    def cannon_fulloffload(self, A, B, C, p, c, alpha, beta, in_place=False):
        """The reference's decompose2D -> multiply -> reorderMatrix on host matrices.  A and B
        are read where they lie when they are column-major doubles already; C is updated in
        place when in_place is set (C must then be a column-major double array), else a copy
        is updated and returned."""
        M = A.shape[0]
        A, B = (np.asfortranarray(x, dtype=np.float64) for x in (A, B))
        if in_place:
            if not (C.flags.f_contiguous and C.dtype == np.float64):
                raise ValueError("in_place needs a column-major float64 C")
        else:
            C = np.array(C, dtype=np.float64, order="F")
        self._check(self.L.ref_cannon_fulloffload(M, p, c, alpha, beta, _ptr(A), _ptr(B), _ptr(C)))
        return C

    def cannon_fulloffload_logged(self, log_dir, A, B, C, p, c, alpha, beta, runs):
        """The reference's fullOffloadSumma25Dgemm with logging on, run in log_dir: returns C
        after `runs` runs; the reference's own CSV log is left in log_dir."""
        M = A.shape[0]
        A, B = (np.array(x, dtype=np.float64, order="F") for x in (A, B))
        C = np.array(C, dtype=np.float64, order="F")
        self._check(self.L.ref_cannon_fulloffload_logged(str(log_dir).encode(), M, p, c, alpha, beta, _ptr(A), _ptr(B),
                                                         _ptr(C), runs))
        return C

    def copy_block(self, rows, cols, src, dst, ldS, ldD, col_major=True):
        """The reference's copyBlock<double> or <float> (by src's dtype) on flat host arrays;
        returns the destination after the copy."""
        src = np.ascontiguousarray(src)
        dst = np.array(dst, dtype=src.dtype)
        fn = self.L.ref_copy_block_f32 if src.dtype == np.float32 else self.L.ref_copy_block_f64
        self._check(fn(rows, cols, src.ctypes.data, dst.ctypes.data, ldS, ldD, int(col_major)))
        return dst

    def cannon_trace(self, p, c):
        pc3 = int((p * p * c / c ** 3) ** 0.5 + 1e-9)
        P = p * p * c
        out = (ctypes.c_int * (P * pc3 * 2))()
        self._check(self.L.ref_cannon_trace(p, c, out))
        return np.array(out, dtype=np.int64).reshape(P, pc3, 2)


_orc_singleton = None
_ref_singleton = None


def orc() -> _Orc:
    global _orc_singleton
    if _orc_singleton is None:
        _orc_singleton = _Orc()
    return _orc_singleton


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref() -> _Ref:
    global _ref_singleton
    if _ref_singleton is None:
        _ref_singleton = _Ref()
    return _ref_singleton


# ---- seeded inputs (numpy PCG64) ---------------------------------------------------------
def uniform(shape, seed, lo=-1.0, hi=1.0):
    """i.i.d. U[lo, hi) doubles, column-major."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.asfortranarray(rng.uniform(lo, hi, size=shape))


def ozaki_matrix(shape, seed, phi):
    """(U[0,1) - 0.5) * exp(phi * N(0,1)), the dynamic-range stress input of the FP64
    emulation configuration (Ozaki/Uchino/Imamura test matrices)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = rng.random(size=shape) - 0.5
    n = rng.standard_normal(size=shape)
    return np.asfortranarray(u * np.exp(phi * n))


def normal32(shape, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.asfortranarray(rng.standard_normal(size=shape, dtype=np.float32))


# ---- FP64 GEMM oracle + error metrics ------------------------------------------------------
def op(X, t):
    return X.T if t.upper() in ("T", "C") else X


def dgemm(A, B, alpha=1.0, beta=0.0, C=None, ta="N", tb="N"):
    """Host FP64 GEMM (OpenBLAS dgemm through numpy): alpha*op(A)@op(B) + beta*C."""
    R = alpha * (op(A, ta) @ op(B, tb))
    if beta != 0.0 and C is not None:
        R = R + beta * C
    return np.asfortranarray(R)


def rel_errors(X, R):
    """(max elementwise relative error with |ref| in the denominator, Frobenius relative
    error).  The reference's Derror (src/Utilities/Validation.cpp:96-99) divides by the
    signed reference value, so negative entries pass trivially; this uses |ref|."""
    X = np.asarray(X, dtype=np.float64)
    R = np.asarray(R, dtype=np.float64)
    d = np.abs(X - R)
    den = np.abs(R)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(den > 0, d / den, d)
    fro = float(np.linalg.norm(d) / max(np.linalg.norm(R), np.finfo(float).tiny))
    return float(rel.max()) if rel.size else 0.0, fro


def digits_of_accuracy(ref_vals, vals):
    """The reference's Dtest_equality digit count (Validation.cpp:57-83), with |a| in the
    denominator instead of the signed a of Derror (:96-99).  Same loop: start at 1e-8,
    tighten by 10x while nothing fails (up to 30 digits); 0 means it failed at 1e-8."""
    ref_vals = np.asarray(ref_vals, dtype=np.float64).ravel()
    vals = np.asarray(vals, dtype=np.float64).ravel()
    d = np.abs(ref_vals - vals)
    den = np.abs(ref_vals)
    err = np.where(ref_vals == 0, d, d / np.where(den == 0, 1, den))
    eps, acc = 1e-8, 8
    failed = bool((err > eps).any())
    while eps > np.finfo(float).tiny and not failed and acc < 30:
        eps *= 0.1
        acc += 1
        failed = bool((err > eps).any())
    return 0 if acc == 8 else acc


# ---- exact restatement of the CRT FP64 emulation (Ozaki scheme II) ------------------------------
# Ozaki, Uchino, Imamura 2025 ("Ozaki Scheme II: A GEMM-oriented emulation of floating-point
# matrix multiplication using an integer modular technique").  The product's path
# (distributed-gemm-thesis_b200/csrc/ozaki2.cu) must agree with this bit for bit for
# alpha = 1, beta = 0 away from subnormal results: the integer product A'B' is exact in both,
# and both round it to FP64 once, to nearest even.
OZAKI2_MODULI = (256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                 223, 217, 211, 199, 197, 193, 191, 181, 179, 173)


def ozaki2_split_residues(y, p: int):
    """The kernels' integer residue split (csrc/crt.cuh ModTable, csrc/ozaki2.cu
    residue_block) restated in numpy: y = a 2^s as float64 (|y| < 2^78), returned as the int8
    symmetric residues of rn(y) modulo p.  Steps: yh = rint(y 2^-40), yl = rint(y - yh 2^40)
    (both exact), 20-bit chunks x0..x3, t = x3 c60 + x2 c40 + x1 c20 + x0 with symmetric
    constants, then the quotient of t + floor(p/2) + 2^21 p by p from one multiply by
    floor(2^38/p) + 1 and a shift, and the low byte of t minus quotient times p."""
    y = np.asarray(y, dtype=np.float64)
    yh = np.rint(y * 2.0 ** -40)
    hi = yh.astype(np.int64)
    lo = np.rint(y - yh * 2.0 ** 40).astype(np.int64)  # exact in float64 (|y - yh 2^40| <= 2^39)
    x0, x1 = lo & 0xFFFFF, lo >> 20
    x2, x3 = hi & 0xFFFFF, hi >> 20

    def sym(v):
        return v - p if v > p // 2 else v

    c20, c40, c60 = sym(2 ** 20 % p), sym(2 ** 40 % p), sym(2 ** 60 % p)
    t = x3 * c60 + x2 * c40 + x1 * c20 + x0
    assert np.all(np.abs(t) < 2 ** 28)
    magic = (1 << 38) // p + 1
    bias = (p // 2 + (p << 21)) * magic
    q = ((t * magic + bias) >> 38).astype(np.int64)
    r = t - q * p
    return (r & 0xFF).astype(np.uint8).view(np.int8)


def _fma(a: float, b: float, c: float) -> float:
    """a b + c rounded once to the nearest double (ties to even): exact rational arithmetic,
    then Python's correctly rounded float()."""
    from fractions import Fraction

    return float(Fraction(a) * Fraction(b) + Fraction(c))


def ozaki2_split_residues_fp64(y, p: int):
    """The kernels' FP64 residue path (csrc/crt.cuh ModTable, the first moduli of
    csrc/ozaki2.cu residue_block) restated step by step with exactly rounded FMAs: yh =
    rint(y 2^-40), yl = rint(y - yh 2^40), t = fma(yh, c40, yl), the low 32-bit words of
    t + 1.5 2^52 and of fma(t, fl(1/p), 1.5 2^52) (t and q = rint(t/p) modulo 2^32), r = their
    32-bit difference t - q p; the int8 byte of r.  Small samples only (pure Python)."""
    import struct

    RINT = 6755399441055744.0
    c40 = float((2 ** 40 % p) - p if 2 ** 40 % p > p // 2 else 2 ** 40 % p)
    out = []
    for v in np.asarray(y, dtype=np.float64).ravel():
        yh = float(np.rint(float(v) * 2.0 ** -40))
        yl = float(np.rint(_fma(-yh, 2.0 ** 40, float(v))))
        t = _fma(yh, c40, yl)
        lo = lambda d: struct.unpack("<q", struct.pack("<d", d))[0] & 0xFFFFFFFF  # the low word
        tl, ql = lo(t + RINT), lo(_fma(t, 1.0 / p, RINT))
        r = (tl - ql * p) & 0xFFFFFFFF
        out.append(((r & 0xFF) ^ 0x80) - 0x80)
    return np.array(out, dtype=np.int8)


def sum3_rn(a: float, b: float, c: float) -> float:
    """The reconstruction's correctly rounded sum of three doubles (csrc/ozaki2.cu sum3_rn,
    Boldo and Melquiond's adder with rounding to odd) restated step by step: two TwoSums, the
    error terms added with rounding to odd (the round-toward-zero sum with its last bit set
    when inexact), one rounding to nearest."""
    import math
    import struct
    from fractions import Fraction

    def two_sum(x, y):
        s = x + y
        bb = s - x
        return s, (x - (s - bb)) + (y - bb)

    def add_round_odd(x, y):
        s, e = two_sum(x, y)
        if e == 0.0:
            return s
        t = s if abs(Fraction(s)) <= abs(Fraction(x) + Fraction(y)) else math.nextafter(s, 0.0)  # toward zero
        bits = struct.unpack("<q", struct.pack("<d", t))[0] | 1
        return struct.unpack("<d", struct.pack("<q", bits))[0]

    uh, ul = two_sum(b, c)
    th, tl = two_sum(a, uh)
    return th + add_round_odd(tl, ul)


def crt_value_fi(residues, nmod: int, limbs: int) -> float:
    """The reconstruction's FP64-limb form with the integer rounding (csrc/ozaki2.cu
    crt_value_fi<L>, before the 2^shift scaling) restated step by step: S_l = sum_j r_j w_jl
    over the B-bit limbs of the CRT weights W_j (B = 41 for 3 limbs, 40 for 4); q =
    rint(S_0 K_0 + S_1 K_1 + ...) with K_l = fl(2^(B l) / fl(P)) and fl(P) accumulated from
    P's 32-bit words as the host code does; d_l = fma(-q, P_l, S_l); carries that leave the
    low digits in [0, 2^B); three 64-bit words of C' in two's complement; the magnitude's top
    word, the word below and a sticky bit for the rest; one correctly rounded conversion.
    Returns C' as the double the kernel hands the scaling.  Pure Python, small samples."""
    import math

    B = 41 if limbs == 3 else 40
    mods = OZAKI2_MODULI[:nmod]
    P = 1
    for p in mods:
        P *= p
    mask = (1 << B) - 1
    S = [0] * limbs
    for r, p in zip(residues, mods):
        M = P // p
        W = M * pow(M % p, -1, p)
        for l in range(limbs):
            S[l] += int(r) * ((W >> (B * l)) & mask)
    pd = 0.0
    for i in reversed(range(6)):  # the host's fl(P): 32-bit words from the top
        pd = pd * 4294967296.0 + float((P >> (32 * i)) & 0xFFFFFFFF)
    K = [math.ldexp(1.0, B * l) / pd for l in range(limbs)]
    xq = float(S[0]) * K[0]
    for l in range(1, limbs):
        xq = _fma(float(S[l]), K[l], xq)
    q = float(round(xq))  # rint: ties to even
    d = [int(_fma(-q, float((P >> (B * l)) & mask), float(S[l]))) for l in range(limbs)]
    for l in range(limbs - 1):
        d[l + 1] += d[l] >> B
        d[l] &= mask
    v = sum(d[l] << (B * l) for l in range(limbs))  # the three words' value, two's complement
    neg = v < 0
    mag = -v if neg else v
    w = [(mag >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(3)]
    ti = 2 if w[2] else (1 if w[1] else 0)
    hi, lo = w[ti], (w[ti - 1] if ti > 0 else 0)
    sticky = ti == 2 and w[0] != 0
    if hi == 0:
        return 0.0
    lz = 64 - hi.bit_length()
    top64 = ((hi << lz) | (lo >> (64 - lz))) & 0xFFFFFFFFFFFFFFFF if lz else hi
    sticky = sticky or (((lo << lz) & 0xFFFFFFFFFFFFFFFF) if lz else lo) != 0
    val = math.ldexp(float(top64 | int(sticky)), 64 * ti - lz)
    return -val if neg else val


def ozaki2_sigmas(nmod: int, k: int):
    """(sigma_A, sigma_B) for nmod moduli and inner dimension k: s = sigma_A + sigma_B is the
    largest with (2^ceil(s/2) + sqrt(k)/2)(2^floor(s/2) + sqrt(k)/2) < (P/2)(1 - 2^-20), checked
    in the log domain with a 1e-9 margin as the kernels' host code does (csrc/ozaki2.cu
    sigma_sum_for); op(A) takes the odd bit."""
    import math

    lg = 0.0
    for p in OZAKI2_MODULI[:nmod]:
        lg += math.log2(float(p))
    t = lg - 1.0 + math.log2(1.0 - 2.0 ** -20)
    r = math.sqrt(float(max(k, 1))) / 2.0
    s = math.floor(t)
    while s > 0:
        a, b = 2.0 ** ((s + 1) // 2), 2.0 ** (s // 2)
        if math.log2((a + r) * (b + r)) < t - 1e-9:
            break
        s -= 1
    return (s + 1) // 2, s // 2


def _row_scale(v, sigma: int):
    """Scale exponent s of one row of op(A) (sigma = sigma_A) or column of op(B) (sigma_B):
    s = sigma - g, where 2^g >= the integer bound of ||v||_2 from q = sum ceil(|v| 2^(20-e))^2,
    e the exponent of max |v| (csrc/ozaki2.cu qnorm_* and row_scale_exp).  No entry cap: the
    scaled row's 2-norm is at most 2^sigma + sqrt(k)/2.  None for a row with inf or NaN."""
    import math

    vals = [abs(float(x)) for x in v]
    if any(not math.isfinite(x) for x in vals):
        return None
    mx = max(vals) if vals else 0.0
    if mx == 0.0:
        return 0
    e = math.frexp(mx)[1]
    q = sum(math.ceil(math.ldexp(x, 20 - e)) ** 2 for x in vals)
    h = ((q - 1).bit_length() + 1) // 2
    return sigma - (e - 20 + h)


def ozaki2_exact(A, B, nmod: int, ta: str = "N", tb: str = "N"):
    """C = op(A) op(B) as the CRT emulation computes it: each row of op(A) / column of op(B)
    scaled by 2^s (so that its 2-norm is at most 2^sigma) and rounded to integers (nearest
    even), their integer product taken exactly, rounded once to FP64 and
    scaled back by 2^-(s_i + t_j).  Pure Python integers: small sizes only."""
    import math

    Aop, Bop = op(A, ta), op(B, tb)
    m, k = Aop.shape
    n = Bop.shape[1]
    sig_a, sig_b = ozaki2_sigmas(nmod, k)
    P = 1
    for p in OZAKI2_MODULI[:nmod]:
        P *= p
    sa = [_row_scale(Aop[i, :], sig_a) for i in range(m)]
    sb = [_row_scale(Bop[:, j], sig_b) for j in range(n)]
    Ai = [[int(round(math.ldexp(float(Aop[i, t]), sa[i]))) for t in range(k)] for i in range(m)]
    Bi = [[int(round(math.ldexp(float(Bop[t, j]), sb[j]))) for t in range(k)] for j in range(n)]
    C = np.empty((m, n))
    for i in range(m):
        for j in range(n):
            exact = sum(a * b for a, b in zip(Ai[i], Bi[j]))
            assert 2 * abs(exact) < P  # the CRT range covers every product (Cauchy-Schwarz bound)
            C[i, j] = math.ldexp(float(exact), -(sa[i] + sb[j]))
    return C


def ozaki2_residue_check(A, B, nmod: int):
    """The CRT identity the kernels rely on, checked in integers: residues of the scaled
    operands in the symmetric ranges, their products reduced mod each p, recombined with
    W_p = (P/p)((P/p)^-1 mod p) and centred, give the exact integer product."""
    import math

    m, k = A.shape
    n = B.shape[1]
    sig_a, sig_b = ozaki2_sigmas(nmod, k)
    mods = OZAKI2_MODULI[:nmod]
    P = math.prod(mods)
    sa = [_row_scale(A[i, :], sig_a) for i in range(m)]
    sb = [_row_scale(B[:, j], sig_b) for j in range(n)]
    Ai = np.array([[int(round(math.ldexp(float(A[i, t]), sa[i]))) for t in range(k)]
                   for i in range(m)], dtype=object)
    Bi = np.array([[int(round(math.ldexp(float(B[t, j]), sb[j]))) for j in range(n)]
                   for t in range(k)], dtype=object)
    # the kernels' integer split takes |x| < 2^78 (every entry is below its row's norm bound)
    assert all(abs(x) <= 2 ** sig_a + math.isqrt(k) for x in Ai.flat)
    assert all(abs(x) <= 2 ** sig_b + math.isqrt(k) for x in Bi.flat)

    def sym(x, p):
        r = x % p
        return r - p if r > (p - 1) // 2 else r

    X = np.zeros((m, n), dtype=object)
    for p in mods:
        ra = np.vectorize(lambda x: sym(x, p), otypes=[np.int64])(Ai)
        rb = np.vectorize(lambda x: sym(x, p), otypes=[np.int64])(Bi)
        assert ra.min() >= -(p // 2) and ra.max() <= (p - 1) // 2
        g = (ra @ rb) % p  # exact in int64 for these sizes
        Mp = P // p
        W = Mp * pow(Mp % p, -1, p)
        X = X + g.astype(object) * W
    X = np.vectorize(lambda x: x % P, otypes=[object])(X)
    X = np.vectorize(lambda x: x - P if x > (P - 1) // 2 else x, otypes=[object])(X)
    return X, Ai.dot(Bi)
