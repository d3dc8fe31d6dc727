"""CPU checks of the C ABI: the library loads, exports every symbol include/dgt.h
declares, and its host-only functions match the oracle.  No kernel runs here."""
import os
import re

import pytest

import dgt
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "dgt.h")).read()
    return sorted(set(re.findall(r"\b(dgt_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = dgt.load()
    names = _declared_symbols()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
    assert {n for n, _, _ in dgt.SIGNATURES} == set(names)


def test_numroc_matches_oracle():
    for n, nb, P in [(15000, 256, 4), (17000, 256, 4), (9000, 256, 4), (4096, 512, 2), (10, 3, 4), (7, 8, 3)]:
        for r in range(P):
            assert dgt.numroc(n, nb, r, 0, P) == O.orc().numroc(n, nb, r, 0, P)


def test_block2d_grid_matches_oracle():
    for P in range(1, 65):
        assert dgt.block2d_grid(P) == O.orc().block2d_grid(P)


@pytest.mark.parametrize("p,c", [(2, 1), (4, 1), (4, 2), (8, 2), (8, 4), (3, 1), (6, 2), (5, 1), (6, 3)])
def test_cannon_schedule(p, c):
    """Reference order when it covers every k-block (bit-identical to the reference's
    trace), shift-by-one order otherwise; either way every stack's steps visit each
    k-block exactly once."""
    for i in range(p):
        for j in range(p):
            seen = []
            for k in range(c):
                mine, covers = dgt.cannon_schedule(p, c, i, j, k)
                ref, ref_covers = O.orc().cannon_schedule(p, c, i, j, k)
                assert covers == ref_covers
                if covers:
                    assert mine == ref
                seen += mine
            assert sorted(seen) == list(range(p))


def test_status_strings():
    lib = dgt.load()
    assert lib.dgt_status_string(0) == b"DGT_SUCCESS"
    assert lib.dgt_status_string(4) == b"DGT_ERROR_TIMEOUT"


def test_header_is_plain_c(tmp_path):
    """include/dgt.h is a C header: a C99 translation unit that includes it compiles with
    -pedantic -Werror (no C++ in the boundary's types or signatures)."""
    import subprocess

    src = tmp_path / "use_dgt.c"
    src.write_text('#include "dgt.h"\nint main(void) { dgt_ipc_handle h; dgt_grid_layout g; (void)h; (void)g; '
                   'return (int)DGT_SUCCESS; }\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    "-c", str(src), "-o", str(tmp_path / "use_dgt.o")], check=True)


def test_new_entries_report_bad_arguments_without_a_device():
    """The boundary returns a status and never aborts: every handle entry given a null handle
    answers DGT_ERROR_NOT_INITIALIZED, and the IPC entries refuse null or empty arguments
    with DGT_ERROR_INVALID_VALUE -- all before any CUDA call, so this runs without a GPU."""
    import ctypes

    lib = dgt.load()
    z = ctypes.c_void_p(0)
    NI = dgt.NOT_INITIALIZED
    assert lib.dgt_copy_block_f32(None, 4, 4, z, z, 4, 4, 1) == NI
    assert lib.dgt_pack_block_cyclic_host(None, 4, 4, 2, 2, 1, 1, z, 4, z, z) == NI
    assert lib.dgt_unpack_block_cyclic_host(None, 4, 4, 2, 2, 1, 1, z, 4, z, z) == NI
    assert lib.dgt_pack_cannon2d_host(None, 4, 2, z, z, z, z, z, z) == NI
    assert lib.dgt_unpack_cannon2d_host(None, 4, 2, z, z) == NI
    assert lib.dgt_pack_block2d_host(None, 4, 4, 4, 2, 1, z, z, z, z, z, z) == NI
    assert lib.dgt_unpack_block2d_host(None, 4, 4, 2, 1, z, z) == NI
    L = dgt.GridLayout(1, 1, 1, 16, 16, 16)
    assert lib.dgt_summa_rank(None, ctypes.byref(L), 0, 4, 4, 4, 1.0, z, z, z, z, 0.0, z, 4, 0, 7) == NI
    assert lib.dgt_cannon25d_rank(None, 4, 1, 1, 0, b"N", b"N", 1.0, z, z, 0.0, z, 0, 7) == NI
    assert lib.dgt_reduce_tiles(None, z, z, 1, 4) == NI
    assert lib.dgt_cannon25d_batch(None, 4, 1, 1, b"N", b"N", 1.0, z, z, 0.0, z, 0, None, 0, 7) == NI
    ptr, h = ctypes.c_void_p(), ctypes.create_string_buffer(64)
    assert lib.dgt_ipc_alloc(0, ctypes.byref(ptr), h) == dgt.INVALID_VALUE
    assert lib.dgt_ipc_alloc(64, None, h) == dgt.INVALID_VALUE
    assert lib.dgt_ipc_open(None, ctypes.byref(ptr)) == dgt.INVALID_VALUE
    assert lib.dgt_ipc_close(None) == dgt.INVALID_VALUE
    assert lib.dgt_ipc_free(None) == dgt.INVALID_VALUE
