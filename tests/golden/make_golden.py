"""Generates the golden fixtures in this folder from the REFERENCE'S OWN CODE.

The reference's layout and 2.5D Cannon sources are compiled by oracle/Makefile against
in-process MPI / host-CUDA test doubles (oracle/_ref/libref.so); this script runs them
on small seeded inputs and stores inputs and outputs as .npz.  It needs the reference
tree at build time, so it runs in the development container only:

    make -C oracle all && python tests/golden/make_golden.py

The GPU box never regenerates these; tests read the committed files.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

PBLAS_CASES = [  # (M, N, Mb, Nb, p, q)
    (10, 7, 3, 2, 2, 2),
    (37, 29, 5, 4, 2, 3),
    (64, 48, 16, 16, 2, 2),
    (100, 90, 7, 11, 3, 4),
    (150, 170, 16, 16, 4, 4),
    (61, 53, 8, 8, 4, 4),
]
BLOCK2D_CASES = [  # (M, N, K, P)
    (10, 12, 7, 4),
    (13, 11, 5, 6),
    (20, 20, 20, 2),  # P=2, M==N: copyBlock's contiguous shortcut hits gatherResult
    (33, 17, 8, 5),
    (16, 24, 9, 9),
]
CANNON_CASES = [(8, 2, 1), (16, 4, 1), (16, 4, 2), (12, 2, 2), (18, 3, 1), (24, 6, 2)]  # (M, p, c)
TRACE_CASES = [(2, 1), (4, 1), (4, 2), (3, 1), (6, 2), (8, 2), (8, 4)]


def main():
    r = O.ref()
    r.use_naive()
    out = {}
    for idx, (M, N, Mb, Nb, p, q) in enumerate(PBLAS_CASES):
        G = O.uniform((M, N), 1000 + idx)
        locs = r.pblas_scatter(G, Mb, Nb, p, q)
        shapes = r.pblas_shapes(M, N, Mb, Nb, p, q)
        back = r.pblas_gather(locs, M, N, Mb, Nb, p, q)
        out[f"pblas{idx}_params"] = np.array([M, N, Mb, Nb, p, q])
        out[f"pblas{idx}_global"] = G
        out[f"pblas{idx}_shapes"] = np.array(shapes)
        out[f"pblas{idx}_locals"] = np.concatenate([l.ravel(order="F") for l in locs])
        # the reference's gather must restore the matrix exactly; store the verdict only
        out[f"pblas{idx}_roundtrip"] = np.array([np.array_equal(back, G)])
    out["numroc_cfg1"] = np.array([r.numroc(4096, 512, i, 0, 2) for i in range(2)])
    out["numroc_cfg2_rows"] = np.array([r.numroc(15000, 256, i, 0, 4) for i in range(4)])
    out["numroc_cfg2_cols"] = np.array([r.numroc(17000, 256, i, 0, 4) for i in range(4)])
    out["numroc_cfg2_k"] = np.array([r.numroc(9000, 256, i, 0, 4) for i in range(4)])
    np.savez_compressed(os.path.join(HERE, "pblas.npz"), **out)

    out = {}
    for idx, (M, N, K, P) in enumerate(BLOCK2D_CASES):
        A, B, C = O.uniform((M, K), 2000 + idx), O.uniform((K, N), 2100 + idx), O.uniform((M, N), 2200 + idx)
        out[f"b2d{idx}_params"] = np.array([M, N, K, P])
        out[f"b2d{idx}_A"], out[f"b2d{idx}_B"], out[f"b2d{idx}_C"] = A, B, C
        dr, dc, _, _ = r.block2d_shapes(M, N, K, P)
        out[f"b2d{idx}_grid"] = np.array([dr, dc])
        for cm in (1, 0):
            lA, lB, lC = r.block2d_deliver(A, B, C, P, bool(cm))
            order = "F" if cm else "C"
            out[f"b2d{idx}_cm{cm}_lA"] = np.concatenate([x.ravel(order=order) for x in lA])
            out[f"b2d{idx}_cm{cm}_lB"] = np.concatenate([x.ravel(order=order) for x in lB])
            out[f"b2d{idx}_cm{cm}_lC"] = np.concatenate([x.ravel(order=order) for x in lC])
            out[f"b2d{idx}_cm{cm}_gathered"] = r.block2d_gather(lC, M, N, K, P, bool(cm))
    np.savez_compressed(os.path.join(HERE, "block2d.npz"), **out)

    out = {}
    for idx, (M, p, c) in enumerate(CANNON_CASES):
        A, B, C = O.uniform((M, M), 3000 + idx), O.uniform((M, M), 3100 + idx), O.uniform((M, M), 3200 + idx)
        lA, lB, lC = r.cannon_decompose(A, B, C, p, c)
        out[f"cannon{idx}_params"] = np.array([M, p, c])
        out[f"cannon{idx}_A"], out[f"cannon{idx}_B"], out[f"cannon{idx}_C"] = A, B, C
        out[f"cannon{idx}_lA"] = np.stack(lA)
        out[f"cannon{idx}_lB"] = np.stack(lB)
        out[f"cannon{idx}_lC"] = np.stack(lC)
        out[f"cannon{idx}_reordered"] = r.cannon_reorder(lC, M, p, c)
        out[f"cannon{idx}_result"] = r.cannon_fulloffload(A, B, C, p, c, 1.5, -0.5)
    for p, c in TRACE_CASES:
        out[f"trace_{p}_{c}"] = r.cannon_trace(p, c)
    np.savez_compressed(os.path.join(HERE, "cannon.npz"), **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
