"""Autotuner through the C ABI: tunes a shape, records the choice, uses it for later
calls (DGT_FP64_AUTO), and round-trips its table through the JSON file."""
import os

import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu


def test_autotune_auto_mode_and_persistence(tmp_path):
    import torch

    m, n, k = 640, 384, 512
    A, B = O.uniform((m, k), 1), O.uniform((k, n), 2)
    dA, dB, dC = dev(A), dev(B), dev(np.zeros((m, n)))
    with dgt.Handle() as h:
        r = h.autotune("N", "N", m, n, k, ptr(dA), m, ptr(dB), k, ptr(dC), m, mode=dgt.FP64_AUTO, tol=1e-14)
        assert r["mode"] in (dgt.FP64_NATIVE, dgt.FP64_OZAKI_INT8, dgt.FP64_OZAKI2_INT8)
        assert r["ms"] > 0
        if r["mode"] == dgt.FP64_OZAKI_INT8:
            assert 4 <= r["slices"] <= 14 and r["rel_diff"] <= 1e-14
        if r["mode"] == dgt.FP64_OZAKI2_INT8:
            assert 10 <= r["slices"] <= 20 and r["rel_diff"] <= 1e-14
        # a later AUTO call uses the recorded choice and stays FP64-accurate
        h.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.0, ptr(dC), m, mode=dgt.FP64_AUTO)
        torch.cuda.synchronize()
        assert O.rel_errors(host(dC, (m, n)), A @ B)[1] <= 1e-13
        path = str(tmp_path / "tune.json")
        h.autotune_save(path)
        text = open(path).read()
        assert "dgt_tuning" in text and text.count("variant") >= 2
    with dgt.Handle() as h2:
        h2.autotune_load(path)
        h2.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.0, ptr(dC), m, mode=dgt.FP64_AUTO)
        torch.cuda.synchronize()
        assert O.rel_errors(host(dC, (m, n)), A @ B)[1] <= 1e-13
        with pytest.raises(dgt.DgtError):
            h2.autotune_load(os.path.join(str(tmp_path), "missing.json"))


def test_autotune_crt_mode_variants():
    """The CRT mode's kernel variants are tuned and the recorded choice is used."""
    import torch

    m, n, k = 512, 640, 768
    A, B = O.uniform((m, k), 3), O.uniform((k, n), 4)
    dA, dB, dC = dev(A), dev(B), dev(np.zeros((m, n)))
    with dgt.Handle() as h:
        h.set_fp64_mode(dgt.FP64_OZAKI2_INT8, 17)
        r = h.autotune("N", "N", m, n, k, ptr(dA), m, ptr(dB), k, ptr(dC), m, mode=dgt.FP64_OZAKI2_INT8)
        assert r["mode"] == dgt.FP64_OZAKI2_INT8 and r["variant"] in (0, 1, 4, 5, 6, 7) and r["slices"] == 17
        h.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.0, ptr(dC), m, mode=dgt.FP64_OZAKI2_INT8, slices=17)
        torch.cuda.synchronize()
        assert O.rel_errors(host(dC, (m, n)), A @ B)[1] <= 1e-15
