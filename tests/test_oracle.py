"""Pins the oracle (oracle/orc.c restatement) against the reference's own code.

Two independent pins:
* golden fixtures in tests/golden/ were produced by running the reference's sources
  (oracle/_ref, see tests/golden/make_golden.py) -- checked here bit for bit;
* when oracle/_ref/libref.so is present, extra seeded shapes run live through both.
"""
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def _split_locals(flat, shapes, order="F"):
    out, off = [], 0
    for r, c in shapes:
        out.append(flat[off:off + r * c].reshape((r, c), order=order))
        off += r * c
    return out


def test_numroc_golden_configs():
    g = _load("pblas.npz")
    o = O.orc()
    assert [o.numroc(4096, 512, i, 0, 2) for i in range(2)] == list(g["numroc_cfg1"])
    assert [o.numroc(15000, 256, i, 0, 4) for i in range(4)] == list(g["numroc_cfg2_rows"])
    assert [o.numroc(17000, 256, i, 0, 4) for i in range(4)] == list(g["numroc_cfg2_cols"])
    assert [o.numroc(9000, 256, i, 0, 4) for i in range(4)] == list(g["numroc_cfg2_k"])
    assert list(g["numroc_cfg2_rows"]) == [3840, 3840, 3736, 3584]
    assert list(g["numroc_cfg2_cols"]) == [4352, 4352, 4200, 4096]


def test_pblas_scatter_gather_golden():
    g = _load("pblas.npz")
    o = O.orc()
    idx = 0
    while f"pblas{idx}_params" in g:
        M, N, Mb, Nb, p, q = (int(v) for v in g[f"pblas{idx}_params"])
        G = g[f"pblas{idx}_global"]
        shapes = [tuple(s) for s in g[f"pblas{idx}_shapes"]]
        assert o.pblas_shapes(M, N, Mb, Nb, p, q) == shapes
        want = _split_locals(g[f"pblas{idx}_locals"], [(r, c) for r, c, _ in shapes])
        got = o.pblas_scatter(G, Mb, Nb, p, q)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
        assert bool(g[f"pblas{idx}_roundtrip"][0])
        assert np.array_equal(o.pblas_gather(got, M, N, Mb, Nb, p, q), G)
        idx += 1
    assert idx >= 5


def test_block2d_golden():
    g = _load("block2d.npz")
    o = O.orc()
    idx = 0
    while f"b2d{idx}_params" in g:
        M, N, K, P = (int(v) for v in g[f"b2d{idx}_params"])
        A, B, C = g[f"b2d{idx}_A"], g[f"b2d{idx}_B"], g[f"b2d{idx}_C"]
        dRow, dCol = o.block2d_grid(P)
        assert [dRow, dCol] == list(g[f"b2d{idx}_grid"])
        tiles = o.block2d_tiles(M, N, K, dRow, dCol)
        for cm in (1, 0):
            order = "F" if cm else "C"
            lA, lB, lC = o.block2d_deliver(A, B, C, P, bool(cm))
            for name, got, shapes in (("lA", lA, [(t[0], K) for t in tiles]), ("lB", lB, [(K, t[1]) for t in tiles]),
                                      ("lC", lC, tiles)):
                want = _split_locals(g[f"b2d{idx}_cm{cm}_{name}"], shapes, order)
                for a, b in zip(got, want):
                    assert np.array_equal(a, b), (idx, cm, name)
            gathered = o.block2d_gather(lC, M, N, P, bool(cm))
            assert np.array_equal(gathered, g[f"b2d{idx}_cm{cm}_gathered"])
        idx += 1
    assert idx >= 4


def test_block2d_gather_reference_quirk_is_reproduced():
    """copyBlock's contiguous shortcut (src/Transfers/sharedTransfers.cpp:51) misplaces
    rank 0's tile in gatherResult when P=2 and M == N (column-major): the reference's
    gathered C is NOT the original C.  The oracle reproduces it; the product does not."""
    g = _load("block2d.npz")
    idx = 2
    assert list(g[f"b2d{idx}_params"]) == [20, 20, 20, 2]
    assert not np.array_equal(g[f"b2d{idx}_cm1_gathered"], g[f"b2d{idx}_C"])
    assert np.array_equal(g[f"b2d{idx}_cm0_gathered"], g[f"b2d{idx}_C"])


def test_cannon_decompose_reorder_golden():
    g = _load("cannon.npz")
    o = O.orc()
    idx = 0
    while f"cannon{idx}_params" in g:
        M, p, c = (int(v) for v in g[f"cannon{idx}_params"])
        A, B, C = g[f"cannon{idx}_A"], g[f"cannon{idx}_B"], g[f"cannon{idx}_C"]
        lA, lB, lC = o.cannon_decompose(A, B, C, p)
        assert np.array_equal(np.stack(lA), g[f"cannon{idx}_lA"])
        assert np.array_equal(np.stack(lB), g[f"cannon{idx}_lB"])
        assert np.array_equal(np.stack(lC), g[f"cannon{idx}_lC"])
        assert np.array_equal(o.cannon_reorder(lC, M, p), g[f"cannon{idx}_reordered"])
        idx += 1


def test_cannon_schedule_matches_reference_trace():
    g = _load("cannon.npz")
    o = O.orc()
    for key in [k for k in g.files if k.startswith("trace_")]:
        _, p, c = key.split("_")
        p, c = int(p), int(c)
        tr = g[key]
        for k in range(c):
            for i in range(p):
                for j in range(p):
                    sched, _ = o.cannon_schedule(p, c, i, j, k)
                    rank = k * p * p + i * p + j
                    assert list(tr[rank, :, 0]) == sched
                    assert list(tr[rank, :, 1]) == sched


def test_cannon_reference_result_and_coverage_bug():
    """The reference's 2.5D Cannon result is alpha*A*B + beta*C when its rotation
    schedule covers every k-block, and wrong otherwise (pc3 >= 3 with colliding
    triangular offsets, e.g. 3x3x1 and 6x6x2)."""
    g = _load("cannon.npz")
    o = O.orc()
    idx = 0
    while f"cannon{idx}_params" in g:
        M, p, c = (int(v) for v in g[f"cannon{idx}_params"])
        A, B, C = g[f"cannon{idx}_A"], g[f"cannon{idx}_B"], g[f"cannon{idx}_C"]
        want = O.dgemm(A, B, 1.5, -0.5, C)
        covers = all(o.cannon_schedule(p, c, i, j, 0)[1] for i in range(p) for j in range(p))
        _, fro = O.rel_errors(g[f"cannon{idx}_result"], want)
        if covers:
            assert fro < 1e-14, (M, p, c, fro)
        else:
            assert fro > 0.1, (M, p, c, fro)
        idx += 1


def test_dd_checker_is_exact_on_integers():
    rng = np.random.default_rng(0)
    A = np.asfortranarray(rng.integers(-1000, 1000, (7, 33)).astype(np.float64))
    B = np.asfortranarray(rng.integers(-1000, 1000, (33, 5)).astype(np.float64))
    C = np.asfortranarray(rng.integers(-9, 9, (7, 5)).astype(np.float64))
    rows, cols = np.meshgrid(np.arange(7), np.arange(5), indexing="ij")
    got = O.orc().dgemm_dd_sample(A, B, 2.0, -3.0, C, rows.ravel(), cols.ravel())
    want = (2.0 * (A @ B) - 3.0 * C).ravel()
    assert np.array_equal(got, want)


def test_digits_metric_uses_abs():
    ref = np.array([-1.0, 2.0])
    assert O.digits_of_accuracy(ref, np.array([-1.5, 2.0])) == 0  # the signed Derror would pass this
    assert O.digits_of_accuracy(ref, ref) == 30


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("case", [(23, 31, 4, 6, 3, 2), (256, 200, 32, 24, 2, 4), (97, 101, 10, 9, 4, 3)])
def test_pblas_live_against_reference(case):
    M, N, Mb, Nb, p, q = case
    G = O.uniform((M, N), 77)
    a = O.orc().pblas_scatter(G, Mb, Nb, p, q)
    b = O.ref().pblas_scatter(G, Mb, Nb, p, q)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert np.array_equal(O.orc().pblas_gather(a, M, N, Mb, Nb, p, q), O.ref().pblas_gather(b, M, N, Mb, Nb, p, q))


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("case", [(31, 29, 13, 6), (40, 40, 40, 2), (17, 23, 5, 7), (64, 48, 32, 8)])
def test_block2d_live_against_reference(case):
    M, N, K, P = case
    A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
    for cm in (True, False):
        a = O.orc().block2d_deliver(A, B, C, P, cm)
        b = O.ref().block2d_deliver(A, B, C, P, cm)
        for xs, ys in zip(a, b):
            for x, y in zip(xs, ys):
                assert np.array_equal(x, y)
        assert np.array_equal(O.orc().block2d_gather(a[2], M, N, P, cm), O.ref().block2d_gather(b[2], M, N, K, P, cm))


def _strided(rows, cols, src, dst, ldS, ldD, col_major=True):
    r, c = (rows, cols) if col_major else (cols, rows)
    out = dst.copy()
    for j in range(c):
        out[j * ldD:j * ldD + r] = src[j * ldS:j * ldS + r]
    return out


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reference_copy_block_instantiations(dtype):
    """The reference's own copyBlock<float> and copyBlock<double> (the float instantiation is
    what dgt_copy_block_f32 replaces) copy a strided block exactly as the strided restatement
    the GPU tests hold the product to, except under their contiguous shortcut
    (sharedTransfers.cpp:51: rows == ldS and columns == ldD after the swap), which copies
    rows*columns contiguous elements whatever ldD is -- reproduced here, fixed in the product."""
    R = O.ref()
    rng = np.random.default_rng(3)
    for rows, cols, ldS, ldD, cm in [(5, 7, 9, 6, True), (64, 3, 64, 64, True), (3, 64, 70, 65, False),
                                     (1, 1, 1, 1, True), (17, 4, 20, 17, True), (4, 17, 20, 19, False)]:
        r, c = (rows, cols) if cm else (cols, rows)
        src = rng.standard_normal(ldS * c).astype(dtype)
        dst = rng.standard_normal(ldD * c).astype(dtype)
        assert np.array_equal(R.copy_block(rows, cols, src, dst, ldS, ldD, cm), _strided(rows, cols, src, dst, ldS, ldD, cm))
    # the shortcut: rows == ldS, cols == ldD, but ldD != rows
    rows, cols, ldS, ldD = 4, 6, 4, 6
    src = rng.standard_normal(ldS * cols).astype(dtype)
    dst = np.zeros(ldD * cols, dtype=dtype)
    got = R.copy_block(rows, cols, src, dst, ldS, ldD, True)
    assert np.array_equal(got[:rows * cols], src[:rows * cols])
    assert not np.array_equal(got, _strided(rows, cols, src, dst, ldS, ldD, True))
