"""CUDA-graph capture of the step schedules: after eager warm-up passes of the sequence
(the first sizes the handle's workspace, the second runs with the final workspace and so
leaves every launch table resident), dgt_dgemm (native, Ozaki slices, and CRT in op(B)
panels on forked side streams), dgt_cannon25d (native: one cooperative launch with the stack
reduction inside; slices: one grouped pass per step), dgt_cannon25d_batch (native and CRT)
and dgt_dgemm_grouped (native and grouped Ozaki) issue only capturable work, so the whole
batch can be captured once and replayed; replay results equal the eager results bit for bit."""
import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, ptr

pytestmark = pytest.mark.gpu


def test_capture_and_replay_all_paths():
    import torch

    m = n = k = 512
    A, B, C = O.uniform((m, k), 1), O.uniform((k, n), 2), O.uniform((m, n), 3)
    dA, dB = dev(A), dev(B)
    outs = {name: dev(C) for name in ("native", "ozaki", "crt_panels")}
    # Cannon 4x4x2 on M = 512
    M, p, c = 512, 4, 2
    lm = M // p
    tA = [dev(O.uniform((lm, lm), 10 + i)) for i in range(p * p)]
    tB = [dev(O.uniform((lm, lm), 40 + i)) for i in range(p * p)]
    tC0 = [O.uniform((lm, lm), 70 + i) for i in range(p * p)]
    tC = [dev(x) for x in tC0]
    tE = [dev(x) for x in tC0]  # the same Cannon, emulated (one grouped Ozaki pass per step)
    # 40 grouped products (device-table path: more than 32 problems)
    rng = np.random.default_rng(0)
    gdesc, gkeep = [], []
    for i in range(40):
        gm, gn, gk = (int(x) for x in rng.integers(1, 300, 3))
        ga, gb, gc = dev(O.uniform((gm, gk), 200 + i)), dev(O.uniform((gk, gn), 300 + i)), dev(O.uniform((gm, gn), 400 + i))
        gkeep.append((ga, gb, gc))
        gdesc.append(dict(m=gm, n=gn, k=gk, alpha=1.0, beta=0.5, A=ptr(ga), lda=gm, B=ptr(gb), ldb=gk, C=ptr(gc), ldc=gm))
    gC0 = [x[2].clone() for x in gkeep]
    # the same products again, emulated in one grouped Ozaki pass (own outputs)
    ekeep = [dev(O.uniform((d["m"], d["n"]), 500 + i)) for i, d in enumerate(gdesc)]
    edesc = [dict(d, C=ptr(c)) for d, c in zip(gdesc, ekeep)]
    eC0 = [x.clone() for x in ekeep]
    # and once more through the CRT scheme's grouped pass
    rkeep = [dev(O.uniform((d["m"], d["n"]), 700 + i)) for i, d in enumerate(gdesc)]
    rdesc = [dict(d, C=ptr(c)) for d, c in zip(gdesc, rkeep)]
    rC0 = [x.clone() for x in rkeep]
    # Cannon plus 6 of the products in one call, native and CRT (own outputs)
    bT = {mode: [dev(x) for x in tC0] for mode in (dgt.FP64_NATIVE, dgt.FP64_OZAKI2_INT8)}
    bkeep = {mode: [dev(O.uniform((d["m"], d["n"]), 900 + i)) for i, d in enumerate(gdesc[:6])] for mode in bT}
    bdesc = {mode: [dict(d, C=ptr(c)) for d, c in zip(gdesc[:6], bkeep[mode])] for mode in bT}
    bC0 = {mode: [x.clone() for x in bkeep[mode]] for mode in bT}

    def batch(h):
        h.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.5, ptr(outs["native"]), m, mode=dgt.FP64_NATIVE)
        h.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.5, ptr(outs["ozaki"]), m, mode=dgt.FP64_OZAKI_INT8,
                slices=7)
        h.cannon25d(M, p, c, 1.0, [ptr(x) for x in tA], [ptr(x) for x in tB], 0.5, [ptr(x) for x in tC])
        h.cannon25d(M, p, c, 1.0, [ptr(x) for x in tA], [ptr(x) for x in tB], 0.5, [ptr(x) for x in tE],
                    mode=dgt.FP64_OZAKI_INT8, slices=7)
        h.dgemm_grouped(gdesc)
        h.dgemm_grouped(edesc, mode=dgt.FP64_OZAKI_INT8, slices=7)
        h.dgemm_grouped(rdesc, mode=dgt.FP64_OZAKI2_INT8, slices=16)
        h.set_tuning(dgt.TUNE_CRT_PANELS, 3)
        h.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.5, ptr(outs["crt_panels"]), m,
                mode=dgt.FP64_OZAKI2_INT8, slices=14)
        h.set_tuning(dgt.TUNE_CRT_PANELS, 0)
        for mode in bT:
            h.cannon25d_batch(M, p, c, 1.0, [ptr(x) for x in tA], [ptr(x) for x in tB], 0.5, [ptr(x) for x in bT[mode]],
                              bdesc[mode], mode=mode, slices=14)

    def reset():
        for name in outs:
            outs[name].copy_(dev(C))
        for x, x0 in zip(tC, tC0):
            x.copy_(dev(x0))
        for x, x0 in zip(tE, tC0):
            x.copy_(dev(x0))
        for x, x0 in zip(gkeep, gC0):
            x[2].copy_(x0)
        for x, x0 in zip(ekeep, eC0):
            x.copy_(x0)
        for x, x0 in zip(rkeep, rC0):
            x.copy_(x0)
        for mode in bT:
            for x, x0 in zip(bT[mode], tC0):
                x.copy_(dev(x0))
            for x, x0 in zip(bkeep[mode], bC0[mode]):
                x.copy_(x0)

    with dgt.Handle() as h:
        side = torch.cuda.Stream()
        h.set_stream(side.cuda_stream)
        with torch.cuda.stream(side):
            batch(h)  # eager: sizes the workspace (calls of different sizes may grow it)
            reset()
            batch(h)  # eager again, now with the final workspace: every table is resident
        torch.cuda.synchronize()
        snap = lambda: ([t.clone() for t in outs.values()] + [x.clone() for x in tC] + [x[2].clone() for x in gkeep] +
                        [x.clone() for x in ekeep] + [x.clone() for x in tE] + [x.clone() for x in rkeep] +
                        [x.clone() for mode in bT for x in bT[mode] + bkeep[mode]])
        eager = snap()
        reset()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            batch(h)
        reset()
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        h.check_device()
        replay = snap()
        for a, b in zip(eager, replay):
            assert torch.equal(a, b)
        # and a second replay after another reset gives the same again
        reset()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(outs["ozaki"], eager[1])
        del g
