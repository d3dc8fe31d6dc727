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
