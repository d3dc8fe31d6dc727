"""The per-rank SUMMA schedule (dgt_summa_schedule: the K segments dgt_summa_rank's GEMM
walks, the same builder dgt_summa runs for every virtual rank), checked on the CPU with
made-up, well-separated base addresses per rank (nothing is dereferenced).  Every segment
is decoded back to (owner rank, global k index) for each of its k columns of A and rows of
B; for every rank the decoded pairs must name each k in 0 .. K-1 exactly once, the A column
and B row of a pair must be the same k, A must come from the rank's process row and B from
its process column (the owners of the panels a SUMMA broadcasts), and runs contiguous in
both owners' buffers must be merged."""
import pytest

import dgt

A_BASE, B_BASE, SPAN = 1 << 40, 80 << 40, 1 << 40


def _decode(seg, p, q, kb, lldA, lldB):
    a, b, lda, ldb, k = seg
    ra, rb = (a - A_BASE) // SPAN, (b - B_BASE) // SPAN
    offa, offb = (a - A_BASE - ra * SPAN) // 8, (b - B_BASE - rb * SPAN) // 8
    assert lda == lldA[ra] and ldb == lldB[rb] and offa % lda == 0
    c0, r0 = offa // lda, offb
    out = []
    for e in range(k):
        c, r = c0 + e, r0 + e
        ka = ((c // kb) * q + ra % q) * kb + c % kb  # A's local column c of process column ra % q
        kb_ = ((r // kb) * p + rb // q) * kb + r % kb  # B's local row r of process row rb // q
        out.append((ra, rb, ka, kb_))
    return out


@pytest.mark.parametrize("p,q,mb,nb,kb,M,N,K", [
    (2, 3, 16, 24, 20, 150, 170, 90), (4, 1, 16, 32, 12, 40, 50, 61), (1, 4, 32, 16, 8, 64, 100, 77),
    (3, 3, 8, 8, 8, 64, 64, 200), (2, 2, 16, 16, 16, 48, 40, 0),
])
def test_summa_schedule_covers_k_once_from_the_owners(p, q, mb, nb, kb, M, N, K):
    P = p * q
    # leading dimensions: local rows (numroc), padded on odd ranks
    lldA = [max(1, dgt.numroc(M, mb, r // q, 0, p)) + (r % 2) for r in range(P)]
    lldB = [max(1, dgt.numroc(K, kb, r // q, 0, p)) + 3 * (r % 2) for r in range(P)]
    A = [A_BASE + r * SPAN for r in range(P)]
    B = [B_BASE + r * SPAN for r in range(P)]
    for rank in range(P):
        i, j = rank // q, rank % q
        segs = dgt.summa_schedule(rank, p, q, mb, nb, kb, M, N, K, A, lldA, B, lldB)
        if K == 0:
            assert segs == [(0, 0, 1, 1, 0)]
            continue
        ks = []
        for seg in segs:
            for ra, rb, ka, kb_ in _decode(seg, p, q, kb, lldA, lldB):
                assert ka == kb_ and ra // q == i and rb % q == j
                ks.append(ka)
        assert sorted(ks) == list(range(K))
        # merging: at most one segment per (A owner, B owner) run of consecutive panels
        assert len(segs) <= -(-K // kb)


def test_summa_schedule_rejects_bad_arguments():
    A, B = [A_BASE], [B_BASE]
    with pytest.raises(dgt.DgtError):
        dgt.summa_schedule(0, 1, 1, 16, 16, 16, 32, 32, 32, A, [8], B, [32])  # lldA < rows
    with pytest.raises(dgt.DgtError):
        dgt.summa_schedule(1, 1, 1, 16, 16, 16, 32, 32, 32, A, [32], B, [32])  # rank outside the grid
