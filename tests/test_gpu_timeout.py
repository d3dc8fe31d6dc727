"""Bounded device waits, exercised without a GPU fault.

Every mbarrier wait in the tensor-core engine and the native TMA / decoupled DMMA kernels,
and the 2.5D Cannon's cross-CTA wait for its stack partials, has a clock64 budget (~2 s).
The test hook DGT_TUNE_TEST_STALL = 1 makes each CTA's producer withhold the operand loads of
its first pipeline stage: a barrier phase that nothing completes, with nothing in flight for
it.  The first wait runs out, the kernel raises its abort flag, drains the loads and MMAs it
did issue, frees TMEM and returns; the host then reads DGT_ERROR_TIMEOUT from
dgt_check_device.  DGT_TUNE_TEST_STALL = 2 keeps the Cannon's partial tiles from counting
themselves, so the stack-0 tiles' wait runs out instead.  With the hook off, the same
handle's next call is exact again.  (The reference has no device-side failure handling: its
*_CHECK macros print and exit, include/errorHandling.hpp:5-56.)"""
import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu


def _stalled_then_exact(h, call, check_result, mode=1):
    import torch

    h.set_tuning(dgt.TUNE_TEST_STALL, mode)
    call()
    torch.cuda.synchronize()  # the kernel returned by itself: the stream drains
    with pytest.raises(dgt.DgtError) as err:
        h.check_device()
    assert err.value.status == dgt.TIMEOUT
    h.check_device()  # the error word was read and cleared
    h.set_tuning(dgt.TUNE_TEST_STALL, 0)
    call()
    torch.cuda.synchronize()
    h.check_device()
    check_result()


@pytest.mark.parametrize("mode,count,variant", [(dgt.FP64_OZAKI2_INT8, 14, 1), (dgt.FP64_OZAKI2_INT8, 14, 4),
                                                (dgt.FP64_OZAKI2_INT8, 14, 5), (dgt.FP64_OZAKI2_INT8, 14, 6),
                                                (dgt.FP64_OZAKI_INT8, 7, 0)])
def test_fp64_emulation_wait_runs_out_then_recovers(mode, count, variant):
    m, n, k = 200, 300, 256
    A, B = O.uniform((m, k), 31), O.uniform((k, n), 32)
    dA, dB, dC = dev(A), dev(B), dev(np.zeros((m, n)))
    with dgt.Handle() as h:
        h.set_tuning(dgt.TUNE_OZAKI_VARIANT, variant)

        def call():
            h.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.0, ptr(dC), m, mode=mode, slices=count)

        def check():
            got = host(dC, (m, n))
            if mode == dgt.FP64_OZAKI2_INT8:
                assert np.array_equal(got, O.ozaki2_exact(A, B, count))
            else:
                assert O.rel_errors(got, O.dgemm(A, B))[1] <= 1e-13

        _stalled_then_exact(h, call, check)


def test_fp32_split_wait_runs_out_then_recovers():
    import torch

    m, n, k = 160, 272, 200
    A, B = O.normal32((m, k), 33), O.normal32((k, n), 34)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    dC = torch.zeros((n, m), dtype=torch.float32, device="cuda")
    with dgt.Handle() as h:

        def call():
            h.sgemm("N", "N", m, n, k, 1.0, dA.data_ptr(), m, dB.data_ptr(), k, 0.0, dC.data_ptr(), m)

        def check():
            got = dC.cpu().numpy().T.astype(np.float64)
            want = A.astype(np.float64) @ B.astype(np.float64)
            assert O.rel_errors(got, want)[1] <= 1e-5

        _stalled_then_exact(h, call, check)


@pytest.mark.parametrize("variant", [14, 18, 23])
def test_native_dmma_wait_runs_out_then_recovers(variant):
    """The native kernels with bounded waits: the TMA kernel (14), the decoupled TMA kernel (18)
    and the decoupled grouped cp.async kernel (23) each stop when their first stage never fills,
    and the handle's next call is exact."""
    m, n, k = 640, 520, 384
    A, B, C = O.uniform((m, k), 41), O.uniform((k, n), 42), O.uniform((m, n), 43)
    dA, dB, dC = dev(A), dev(B), dev(C)
    with dgt.Handle() as h:
        h.set_tuning(dgt.TUNE_DMMA_VARIANT, variant)

        def call():
            dC.copy_(dev(C))
            h.dgemm("N", "N", m, n, k, 1.5, ptr(dA), m, ptr(dB), k, -0.5, ptr(dC), m, mode=dgt.FP64_NATIVE)

        def check():
            assert O.rel_errors(host(dC, (m, n)), O.dgemm(A, B, 1.5, -0.5, C))[1] <= 1e-13

        _stalled_then_exact(h, call, check)


@pytest.mark.parametrize("variant", [2, 23])
def test_stack_reduction_wait_runs_out_then_recovers(variant):
    """The native 2.5D Cannon's one launch: when no partial tile counts itself, the stack-0
    tiles' bounded wait for them runs out (one budget for the whole launch), the launch
    returns, dgt_check_device reports DGT_ERROR_TIMEOUT, and the next call is exact."""
    import torch

    M, p, c = 512, 4, 2
    lm = M // p
    A, B, C = O.uniform((M, M), 51), O.uniform((M, M), 52), O.uniform((M, M), 53)
    dA, dB, dC = dev(A), dev(B), dev(C)
    mk = lambda: [torch.zeros((lm, lm), dtype=torch.float64, device="cuda") for _ in range(p * p)]
    tA, tB, tC = mk(), mk(), mk()
    with dgt.Handle() as h:
        h.set_tuning(dgt.TUNE_DMMA_VARIANT, variant)
        h.pack_cannon2d(M, p, ptr(dA), ptr(dB), ptr(dC), [ptr(x) for x in tA], [ptr(x) for x in tB],
                        [ptr(x) for x in tC])
        C0 = [x.clone() for x in tC]

        def call():
            for x, x0 in zip(tC, C0):
                x.copy_(x0)
            h.cannon25d(M, p, c, 1.0, [ptr(x) for x in tA], [ptr(x) for x in tB], 0.5, [ptr(x) for x in tC])

        def check():
            out = dev(np.zeros((M, M)))
            h.unpack_cannon2d(M, p, ptr(out), [ptr(x) for x in tC])
            torch.cuda.synchronize()
            assert O.rel_errors(host(out, (M, M)), O.dgemm(A, B, 1.0, 0.5, C))[1] <= 1e-13

        _stalled_then_exact(h, call, check, mode=2)
