"""Python view of libdgt's C ABI (include/dgt.h) through ctypes.

The binding passes raw device pointers and sizes, exactly what a C, C++ or Fortran
caller of the library would pass; torch is used by callers only to own device memory
and streams.  Every non-success status raises DgtError.  There is no fallback: if the
CUDA library is missing, loading fails loudly.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libdgt.so")

SUCCESS, INVALID_VALUE, UNSUPPORTED, CUDA_ERROR, TIMEOUT, ALLOC, NOT_INITIALIZED = range(7)
FP64_NATIVE, FP64_OZAKI_INT8, FP64_OZAKI_BF16, FP64_AUTO, FP64_OZAKI2_INT8 = range(5)
FP32_SIMT, FP32_BF16X1, FP32_BF16X3 = range(3)
TUNE_DMMA_VARIANT, TUNE_OZAKI_SLICES, TUNE_PROFILE, TUNE_OZAKI_VARIANT, TUNE_TEST_STALL, TUNE_FUSE_STEPS, \
    TUNE_CRT_PANELS = range(7)

_c_i64 = ctypes.c_int64
_c_i32 = ctypes.c_int32
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


class DgtError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {msg}")


_STATUS_NAMES = {0: "DGT_SUCCESS", 1: "DGT_ERROR_INVALID_VALUE", 2: "DGT_ERROR_UNSUPPORTED", 3: "DGT_ERROR_CUDA",
                 4: "DGT_ERROR_TIMEOUT", 5: "DGT_ERROR_ALLOC", 6: "DGT_ERROR_NOT_INITIALIZED"}


class GemmDesc(ctypes.Structure):
    _fields_ = [("m", _c_i64), ("n", _c_i64), ("k", _c_i64), ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
                ("A", _vp), ("lda", _c_i64), ("B", _vp), ("ldb", _c_i64), ("C", _vp), ("ldc", _c_i64),
                ("transa", ctypes.c_char), ("transb", ctypes.c_char)]


class TuneResult(ctypes.Structure):
    _fields_ = [("mode", _c_i32), ("variant", _c_i32), ("slices", _c_i32), ("ms", ctypes.c_float),
                ("rel_diff", ctypes.c_double)]


class GridLayout(ctypes.Structure):
    _fields_ = [("p", _c_i32), ("q", _c_i32), ("c", _c_i32), ("mb", _c_i64), ("nb", _c_i64), ("kb", _c_i64)]


# (name, restype, argtypes) for every symbol include/dgt.h declares
SIGNATURES = [
    ("dgt_create", _c_i32, [ctypes.POINTER(_vp)]),
    ("dgt_destroy", _c_i32, [_vp]),
    ("dgt_set_stream", _c_i32, [_vp, _vp]),
    ("dgt_get_stream", _c_i32, [_vp, ctypes.POINTER(_vp)]),
    ("dgt_set_fp64_mode", _c_i32, [_vp, _c_i32, ctypes.c_int]),
    ("dgt_status_string", ctypes.c_char_p, [_c_i32]),
    ("dgt_last_error", ctypes.c_char_p, [_vp]),
    ("dgt_check_device", _c_i32, [_vp]),
    ("dgt_dgemm", _c_i32, [_vp, ctypes.c_char, ctypes.c_char, _c_i64, _c_i64, _c_i64, _dp, _vp, _c_i64, _vp, _c_i64,
                           _dp, _vp, _c_i64]),
    ("dgt_dgemm_ex", _c_i32, [_vp, ctypes.c_char, ctypes.c_char, _c_i64, _c_i64, _c_i64, _dp, _vp, _c_i64, _vp,
                              _c_i64, _dp, _vp, _c_i64, _c_i32, ctypes.c_int]),
    ("dgt_dgemm_workspace_size", _c_i32, [_c_i64, _c_i64, _c_i64, _c_i32, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_size_t)]),
    ("dgt_dgemm_host", _c_i32, [_vp, ctypes.c_char, ctypes.c_char, _c_i64, _c_i64, _c_i64, _dp, _vp, _c_i64, _vp,
                                _c_i64, _dp, _vp, _c_i64, _c_i32, ctypes.c_int, _c_i64]),
    ("dgt_sgemm", _c_i32, [_vp, ctypes.c_char, ctypes.c_char, _c_i64, _c_i64, _c_i64, _fp, _vp, _c_i64, _vp, _c_i64,
                           _fp, _vp, _c_i64, _c_i32]),
    ("dgt_dgemm_grouped", _c_i32, [_vp, ctypes.c_int, ctypes.POINTER(GemmDesc), _c_i32, ctypes.c_int]),
    ("dgt_numroc", _c_i32, [_c_i32] * 5),
    ("dgt_block2d_grid", _c_i32, [_c_i32, ctypes.POINTER(_c_i32), ctypes.POINTER(_c_i32)]),
    ("dgt_summa", _c_i32, [_vp, ctypes.POINTER(GridLayout), _c_i64, _c_i64, _c_i64, ctypes.c_double, _vp, _vp, _vp,
                           _vp, ctypes.c_double, _vp, _vp, _c_i32, ctypes.c_int]),
    ("dgt_summa_rank", _c_i32, [_vp, ctypes.POINTER(GridLayout), _c_i32, _c_i64, _c_i64, _c_i64, ctypes.c_double,
                                _vp, _vp, _vp, _vp, ctypes.c_double, _vp, _c_i64, _c_i32, ctypes.c_int]),
    ("dgt_cannon25d_rank", _c_i32, [_vp, _c_i64, _c_i32, _c_i32, _c_i32, ctypes.c_char, ctypes.c_char,
                                    ctypes.c_double, _vp, _vp, ctypes.c_double, _vp, _c_i32, ctypes.c_int]),
    ("dgt_reduce_tiles", _c_i32, [_vp, _vp, _vp, _c_i32, _c_i64]),
    ("dgt_ipc_alloc", _c_i32, [ctypes.c_size_t, ctypes.POINTER(_vp), ctypes.c_char_p]),
    ("dgt_ipc_open", _c_i32, [ctypes.c_char_p, ctypes.POINTER(_vp)]),
    ("dgt_ipc_close", _c_i32, [_vp]),
    ("dgt_ipc_free", _c_i32, [_vp]),
    ("dgt_summa_schedule", _c_i32, [ctypes.POINTER(GridLayout), _c_i32, _c_i64, _c_i64, _c_i64, _vp, _vp, _vp, _vp,
                                    _vp, _c_i32]),
    ("dgt_cannon25d", _c_i32, [_vp, _c_i64, _c_i32, _c_i32, ctypes.c_char, ctypes.c_char, ctypes.c_double, _vp, _vp,
                               ctypes.c_double, _vp, _c_i32, ctypes.c_int]),
    ("dgt_cannon25d_batch", _c_i32, [_vp, _c_i64, _c_i32, _c_i32, ctypes.c_char, ctypes.c_char, ctypes.c_double,
                                     _vp, _vp, ctypes.c_double, _vp, _c_i32, ctypes.POINTER(GemmDesc), _c_i32,
                                     ctypes.c_int]),
    ("dgt_cannon_schedule", _c_i32, [_c_i32] * 5 + [ctypes.POINTER(_c_i32)]),
    ("dgt_pack_block_cyclic", _c_i32, [_vp, _c_i64, _c_i64, _c_i64, _c_i64, _c_i32, _c_i32, _vp, _c_i64, _vp, _vp]),
    ("dgt_unpack_block_cyclic", _c_i32, [_vp, _c_i64, _c_i64, _c_i64, _c_i64, _c_i32, _c_i32, _vp, _c_i64, _vp,
                                         _vp]),
    ("dgt_pack_block_cyclic_host", _c_i32, [_vp, _c_i64, _c_i64, _c_i64, _c_i64, _c_i32, _c_i32, _vp, _c_i64, _vp,
                                            _vp]),
    ("dgt_unpack_block_cyclic_host", _c_i32, [_vp, _c_i64, _c_i64, _c_i64, _c_i64, _c_i32, _c_i32, _vp, _c_i64,
                                              _vp, _vp]),
    ("dgt_pack_cannon2d_host", _c_i32, [_vp, _c_i64, _c_i32, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("dgt_unpack_cannon2d_host", _c_i32, [_vp, _c_i64, _c_i32, _vp, _vp]),
    ("dgt_pack_block2d_host", _c_i32, [_vp, _c_i64, _c_i64, _c_i64, _c_i32, _c_i32, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("dgt_unpack_block2d_host", _c_i32, [_vp, _c_i64, _c_i64, _c_i32, _c_i32, _vp, _vp]),
    ("dgt_pack_block2d", _c_i32, [_vp, _c_i64, _c_i64, _c_i64, _c_i32, _c_i32, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("dgt_unpack_block2d", _c_i32, [_vp, _c_i64, _c_i64, _c_i32, _c_i32, _vp, _vp]),
    ("dgt_pack_cannon2d", _c_i32, [_vp, _c_i64, _c_i32, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("dgt_unpack_cannon2d", _c_i32, [_vp, _c_i64, _c_i32, _vp, _vp]),
    ("dgt_copy_block", _c_i32, [_vp, _c_i64, _c_i64, _vp, _vp, _c_i64, _c_i64, _c_i32]),
    ("dgt_copy_block_f32", _c_i32, [_vp, _c_i64, _c_i64, _vp, _vp, _c_i64, _c_i64, _c_i32]),
    ("dgt_set_tuning", _c_i32, [_vp, _c_i32, _c_i32]),
    ("dgt_get_tuning", _c_i32, [_vp, _c_i32, ctypes.POINTER(_c_i32)]),
    ("dgt_autotune_dgemm", _c_i32, [_vp, ctypes.c_char, ctypes.c_char, _c_i64, _c_i64, _c_i64, _vp, _c_i64, _vp,
                                     _c_i64, _vp, _c_i64, _c_i32, ctypes.c_double, ctypes.POINTER(TuneResult)]),
    ("dgt_autotune_save", _c_i32, [_vp, ctypes.c_char_p]),
    ("dgt_autotune_load", _c_i32, [_vp, ctypes.c_char_p]),
    ("dgt_probe_peak", _c_i32, [_vp, _c_i32, _dp]),
    ("dgt_last_timings", _c_i32, [_vp, ctypes.POINTER(ctypes.c_float), _c_i32]),
    ("dgt_launch_count", _c_i64, [_vp]),
    ("dgt_dgemm_ozaki_static", _c_i32, [_vp, ctypes.c_char, ctypes.c_char, _c_i64, _c_i64, _c_i64, _dp, _vp, _c_i64,
                                         _vp, _c_i64, _dp, _vp, _c_i64, _c_i32]),
    ("dgt_ozaki_static_check", _c_i32, [_vp]),
]

_lib = None


def load(path: str = LIB_PATH):
    """Loads libdgt.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"libdgt.so not found at {path}; run __graft_entry__.build() or make -C "
                          f"distributed-gemm-thesis_b200")
        lib = ctypes.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _ptrs(ptrs):
    arr = (_vp * len(ptrs))(*[int(p) for p in ptrs])
    return arr


def _i64s(vals):
    return (_c_i64 * len(vals))(*[int(v) for v in vals])


def dgemm_workspace_size(m, n, k, mode=FP64_NATIVE, slices=7):
    """dgt_dgemm_workspace_size: device workspace bytes a dgt_dgemm_ex call of this shape needs
    (an upper bound over kernel variants); no handle, no device call."""
    out = ctypes.c_size_t()
    st = load().dgt_dgemm_workspace_size(m, n, k, mode, slices, ctypes.byref(out))
    if st != 0:
        raise DgtError(st, "dgt_dgemm_workspace_size")
    return out.value


class Handle:
    """Owns one dgt_handle_t.  `stream` is a raw cudaStream_t value (0 = legacy default)."""

    def __init__(self, stream: int = 0):
        self.lib = load()
        h = _vp()
        self._check(self.lib.dgt_create(ctypes.byref(h)))
        self.h = h
        if stream:
            self._check(self.lib.dgt_set_stream(self.h, _vp(stream)))

    def _check(self, st):
        if st != SUCCESS:
            msg = self.lib.dgt_last_error(self.h).decode() if getattr(self, "h", None) else ""
            raise DgtError(st, msg)

    def close(self):
        if getattr(self, "h", None):
            self.lib.dgt_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- control --------------------------------------------------------------------
    def set_stream(self, stream: int):
        self._check(self.lib.dgt_set_stream(self.h, _vp(stream)))

    def set_fp64_mode(self, mode: int, slices: int = 7):
        self._check(self.lib.dgt_set_fp64_mode(self.h, mode, slices))

    def check_device(self):
        self._check(self.lib.dgt_check_device(self.h))

    def launch_count(self) -> int:
        return int(self.lib.dgt_launch_count(self.h))

    def set_tuning(self, knob: int, value: int):
        self._check(self.lib.dgt_set_tuning(self.h, knob, value))

    def get_tuning(self, knob: int) -> int:
        v = _c_i32()
        self._check(self.lib.dgt_get_tuning(self.h, knob, ctypes.byref(v)))
        return v.value

    def last_timings(self):
        """(split_ms, gemm_ms) of the last GEMM call; needs set_tuning(TUNE_PROFILE, 1)."""
        out = (ctypes.c_float * 2)()
        n = self.lib.dgt_last_timings(self.h, out, 2)
        return (out[0], out[1]) if n == 2 else (None, None)

    def autotune(self, ta, tb, m, n, k, A, lda, B, ldb, C, ldc, mode=FP64_AUTO, tol=1e-14):
        r = TuneResult()
        self._check(self.lib.dgt_autotune_dgemm(self.h, ta.encode(), tb.encode(), m, n, k, _vp(A), lda, _vp(B), ldb,
                                                _vp(C), ldc, mode, tol, ctypes.byref(r)))
        return {"mode": r.mode, "variant": r.variant, "slices": r.slices, "ms": r.ms, "rel_diff": r.rel_diff}

    def autotune_save(self, path):
        self._check(self.lib.dgt_autotune_save(self.h, path.encode()))

    def autotune_load(self, path):
        self._check(self.lib.dgt_autotune_load(self.h, path.encode()))

    def probe_peak(self, kind: int) -> float:
        v = ctypes.c_double()
        self._check(self.lib.dgt_probe_peak(self.h, kind, ctypes.byref(v)))
        return v.value

    # -- GEMM -------------------------------------------------------------------------
    def dgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, mode=None, slices=7):
        a, b = ctypes.c_double(alpha), ctypes.c_double(beta)
        if mode is None:
            st = self.lib.dgt_dgemm(self.h, ta.encode(), tb.encode(), m, n, k, ctypes.byref(a), _vp(A), lda, _vp(B),
                                    ldb, ctypes.byref(b), _vp(C), ldc)
        else:
            st = self.lib.dgt_dgemm_ex(self.h, ta.encode(), tb.encode(), m, n, k, ctypes.byref(a), _vp(A), lda,
                                       _vp(B), ldb, ctypes.byref(b), _vp(C), ldc, mode, slices)
        self._check(st)

    def dgemm_host(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, mode=FP64_NATIVE, slices=7,
                   panel_cols=0):
        """dgt_dgemm_host: A, B, C are HOST addresses (page-locked for overlapped copies)."""
        a, b = ctypes.c_double(alpha), ctypes.c_double(beta)
        self._check(self.lib.dgt_dgemm_host(self.h, ta.encode(), tb.encode(), m, n, k, ctypes.byref(a), _vp(A), lda,
                                            _vp(B), ldb, ctypes.byref(b), _vp(C), ldc, mode, slices, panel_cols))

    def sgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, mode=FP32_BF16X3):
        a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
        self._check(self.lib.dgt_sgemm(self.h, ta.encode(), tb.encode(), m, n, k, ctypes.byref(a), _vp(A), lda,
                                       _vp(B), ldb, ctypes.byref(b), _vp(C), ldc, mode))

    @staticmethod
    def _desc_array(descs):
        arr = (GemmDesc * max(1, len(descs)))()
        for i, d in enumerate(descs):
            arr[i] = GemmDesc(d["m"], d["n"], d["k"], d.get("alpha", 1.0), d.get("beta", 0.0), d["A"], d["lda"],
                              d["B"], d["ldb"], d["C"], d["ldc"], d.get("transa", "N").encode(),
                              d.get("transb", "N").encode())
        return arr

    def dgemm_grouped(self, descs, mode=FP64_NATIVE, slices=7):
        self._check(self.lib.dgt_dgemm_grouped(self.h, len(descs), self._desc_array(descs), mode, slices))

    def summa(self, p, q, mb, nb, kb, M, N, K, alpha, A_locals, lldA, B_locals, lldB, beta, C_locals, lldC,
              mode=FP64_NATIVE, slices=7):
        L = GridLayout(p, q, 1, mb, nb, kb)
        self._check(self.lib.dgt_summa(self.h, ctypes.byref(L), M, N, K, alpha, _ptrs(A_locals), _i64s(lldA),
                                       _ptrs(B_locals), _i64s(lldB), beta, _ptrs(C_locals), _i64s(lldC), mode,
                                       slices))

    def summa_rank(self, rank, p, q, mb, nb, kb, M, N, K, alpha, A_locals, lldA, B_locals, lldB, beta, C, ldc,
                   mode=FP64_NATIVE, slices=7):
        """Rank `rank`'s C block of the SUMMA; A_locals / B_locals may be peer-mapped pointers."""
        L = GridLayout(p, q, 1, mb, nb, kb)
        self._check(self.lib.dgt_summa_rank(self.h, ctypes.byref(L), rank, M, N, K, alpha, _ptrs(A_locals),
                                            _i64s(lldA), _ptrs(B_locals), _i64s(lldB), beta, _vp(C), ldc, mode,
                                            slices))

    def cannon25d_rank(self, M, p, c, rank, alpha, A_tiles, B_tiles, beta, C_tile, ta="N", tb="N",
                       mode=FP64_NATIVE, slices=7):
        """Rank `rank`'s stack partial of the 2.5D Cannon; A_tiles / B_tiles may be peer-mapped."""
        self._check(self.lib.dgt_cannon25d_rank(self.h, M, p, c, rank, ta.encode(), tb.encode(), alpha,
                                                _ptrs(A_tiles), _ptrs(B_tiles), beta, _vp(C_tile), mode, slices))

    def reduce_tiles(self, C, parts, elems):
        """C[e] += sum of parts[s][e], in order (parts may be peer-mapped)."""
        self._check(self.lib.dgt_reduce_tiles(self.h, _vp(C), _ptrs(parts), len(parts), elems))

    def cannon25d(self, M, p, c, alpha, A_tiles, B_tiles, beta, C_tiles, ta="N", tb="N", mode=FP64_NATIVE,
                  slices=7):
        self._check(self.lib.dgt_cannon25d(self.h, M, p, c, ta.encode(), tb.encode(), alpha, _ptrs(A_tiles),
                                           _ptrs(B_tiles), beta, _ptrs(C_tiles), mode, slices))

    def cannon25d_batch(self, M, p, c, alpha, A_tiles, B_tiles, beta, C_tiles, descs, ta="N", tb="N",
                        mode=FP64_NATIVE, slices=7):
        """The 2.5D Cannon multiply plus the grouped products `descs` in one grouped launch."""
        self._check(self.lib.dgt_cannon25d_batch(self.h, M, p, c, ta.encode(), tb.encode(), alpha, _ptrs(A_tiles),
                                                 _ptrs(B_tiles), beta, _ptrs(C_tiles), len(descs),
                                                 self._desc_array(descs), mode, slices))

    # -- layout ----------------------------------------------------------------------------
    def pack_block_cyclic(self, M, N, mb, nb, p, q, G, ldg, locals_, lld):
        self._check(self.lib.dgt_pack_block_cyclic(self.h, M, N, mb, nb, p, q, _vp(G), ldg, _ptrs(locals_),
                                                   _i64s(lld)))

    def unpack_block_cyclic(self, M, N, mb, nb, p, q, G, ldg, locals_, lld):
        self._check(self.lib.dgt_unpack_block_cyclic(self.h, M, N, mb, nb, p, q, _vp(G), ldg, _ptrs(locals_),
                                                     _i64s(lld)))

    def pack_block_cyclic_host(self, M, N, mb, nb, p, q, G, ldg, locals_, lld):
        """Scatter from a page-locked host global matrix in one pass (no device copy of G)."""
        self._check(self.lib.dgt_pack_block_cyclic_host(self.h, M, N, mb, nb, p, q, _vp(G), ldg, _ptrs(locals_),
                                                        _i64s(lld)))

    def unpack_block_cyclic_host(self, M, N, mb, nb, p, q, G, ldg, locals_, lld):
        self._check(self.lib.dgt_unpack_block_cyclic_host(self.h, M, N, mb, nb, p, q, _vp(G), ldg, _ptrs(locals_),
                                                          _i64s(lld)))

    def pack_cannon2d_host(self, M, p, A, B, C, lA, lB, lC):
        """decompose2D from page-locked host A, B, C in one pass."""
        self._check(self.lib.dgt_pack_cannon2d_host(self.h, M, p, _vp(A), _vp(B), _vp(C), _ptrs(lA), _ptrs(lB),
                                                    _ptrs(lC)))

    def unpack_cannon2d_host(self, M, p, C, lC):
        self._check(self.lib.dgt_unpack_cannon2d_host(self.h, M, p, _vp(C), _ptrs(lC)))

    def pack_block2d_host(self, M, N, K, P, col_major, A, B, C, lA, lB, lC):
        """deliverMatrix from page-locked host A, B, C in one pass."""
        self._check(self.lib.dgt_pack_block2d_host(self.h, M, N, K, P, int(col_major), _vp(A), _vp(B), _vp(C),
                                                   _ptrs(lA), _ptrs(lB), _ptrs(lC)))

    def unpack_block2d_host(self, M, N, P, col_major, C, lC):
        self._check(self.lib.dgt_unpack_block2d_host(self.h, M, N, P, int(col_major), _vp(C), _ptrs(lC)))

    def pack_block2d(self, M, N, K, P, col_major, A, B, C, lA, lB, lC):
        self._check(self.lib.dgt_pack_block2d(self.h, M, N, K, P, int(col_major), _vp(A), _vp(B), _vp(C), _ptrs(lA),
                                              _ptrs(lB), _ptrs(lC)))

    def unpack_block2d(self, M, N, P, col_major, C, lC):
        self._check(self.lib.dgt_unpack_block2d(self.h, M, N, P, int(col_major), _vp(C), _ptrs(lC)))

    def pack_cannon2d(self, M, p, A, B, C, lA, lB, lC):
        self._check(self.lib.dgt_pack_cannon2d(self.h, M, p, _vp(A), _vp(B), _vp(C), _ptrs(lA), _ptrs(lB),
                                               _ptrs(lC)))

    def unpack_cannon2d(self, M, p, C, lC):
        self._check(self.lib.dgt_unpack_cannon2d(self.h, M, p, _vp(C), _ptrs(lC)))

    def copy_block(self, rows, cols, src, dst, ldS, ldD, col_major=True):
        self._check(self.lib.dgt_copy_block(self.h, rows, cols, _vp(src), _vp(dst), ldS, ldD, int(col_major)))

    def copy_block_f32(self, rows, cols, src, dst, ldS, ldD, col_major=True):
        """copyBlock<float>: the same strided copy on 4-byte elements."""
        self._check(self.lib.dgt_copy_block_f32(self.h, rows, cols, _vp(src), _vp(dst), ldS, ldD, int(col_major)))


def numroc(n, nb, iproc, isrproc, nprocs) -> int:
    return int(load().dgt_numroc(n, nb, iproc, isrproc, nprocs))


def block2d_grid(P):
    a, b = _c_i32(), _c_i32()
    st = load().dgt_block2d_grid(P, ctypes.byref(a), ctypes.byref(b))
    if st != SUCCESS:
        raise DgtError(st, "block2d_grid")
    return a.value, b.value


def summa_schedule(rank, p, q, mb, nb, kb, M, N, K, A_locals, lldA, B_locals, lldB):
    """[(A address, B address, lda, ldb, k), ...]: the K segments rank `rank`'s SUMMA GEMM
    walks (host only; the addresses are not dereferenced)."""
    lib = load()
    L = GridLayout(p, q, 1, mb, nb, kb)
    args = (ctypes.byref(L), rank, M, N, K, _ptrs(A_locals), _i64s(lldA), _ptrs(B_locals), _i64s(lldB))
    n = lib.dgt_summa_schedule(*args, None, 0)
    if n < 0:
        raise DgtError(INVALID_VALUE, "dgt_summa_schedule")
    out = (ctypes.c_int64 * (5 * max(n, 1)))()
    lib.dgt_summa_schedule(*args, out, n)
    return [tuple(out[5 * s:5 * s + 5]) for s in range(n)]


def cannon_schedule(p, c, i, j, k):
    out = (_c_i32 * max(p // c, 1))()
    covers = load().dgt_cannon_schedule(p, c, i, j, k, out)
    if covers < 0:
        raise DgtError(INVALID_VALUE, "cannon_schedule")
    return list(out)[: p // c], bool(covers)
