// Host-buffer GEMM (dgt_dgemm_host): C = alpha op(A) op(B) + beta C with A, B and C in host
// memory.  The reference's drivers bring host blocks to the device and back around each
// local GEMM with plain copies (src/Tests/summa25Dtest.cpp:85-94,
// src/Wrappers/cuBLASMp/cuBLASMpWrapped.cpp:104-106), so the copies and the GEMM run one
// after the other.  Here op(A) goes to the device once, op(B) and C travel in column panels,
// and three streams overlap them:
//
//   copy-in stream : A | B_0 (C_0) | B_1 (C_1) | B_2 ...
//   handle stream  :     [A split] | panel 0   | panel 1   | ...
//   copy-out stream:                            | C_0 out   | C_1 out ...
//
// Two device buffers per panel operand alternate, guarded by events (a B buffer is refilled
// once its panel has been split or multiplied, a C buffer once its result has left).  In the
// CRT mode op(A) is split into residue planes once and every panel runs only its own split,
// residue GEMM and reconstruction; since row scaling depends on op(A)'s rows alone and column
// scaling on op(B)'s columns alone, each panel's result equals the corresponding columns of
// the whole-matrix call bit for bit.  Other modes run the device GEMM per panel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "crt.cuh"
#include "dgt_internal.cuh"

using namespace dgt;

namespace {

enum {
    EV_START, EV_A, EV_IN0, EV_IN1, EV_BFREE0, EV_BFREE1, EV_C0, EV_C1, EV_OUT0, EV_OUT1, EV_JOIN_IN, EV_JOIN_OUT,
    EV_COUNT
};
static_assert(EV_COUNT <= 12, "dgt_context::copy_ev holds 12 events");

// Once copies may be queued, every exit (success or error) orders the handle's stream after
// all work of both copy streams, so nothing of this call can still be writing the handle's
// workspace or the caller's C when the next work on the handle's stream starts.
struct JoinCopyStreams {
    cudaStream_t s = nullptr, si = nullptr, so = nullptr;
    cudaEvent_t ei = nullptr, eo = nullptr;
    bool armed = false;
    ~JoinCopyStreams() {
        if (!armed) return;
        cudaEventRecord(ei, si);
        cudaEventRecord(eo, so);
        cudaStreamWaitEvent(s, ei, 0);
        cudaStreamWaitEvent(s, eo, 0);
    }
};

dgt_status ensure_copy_streams(dgt_context* h) {
    for (auto& cs : h->copy_stream)
        if (!cs) DGT_CUDA_TRY(h, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    for (int i = 0; i < EV_COUNT; ++i)
        if (!h->copy_ev[i]) DGT_CUDA_TRY(h, cudaEventCreateWithFlags(&h->copy_ev[i], cudaEventDisableTiming));
    return DGT_SUCCESS;
}

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

extern "C" dgt_status dgt_dgemm_host(dgt_handle_t h, char transa, char transb, int64_t m, int64_t n, int64_t k,
                                     const double* alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
                                     const double* beta, double* C, int64_t ldc, dgt_fp64_mode mode, int slices,
                                     int64_t panel_cols) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (!alpha || !beta) return fail(h, DGT_ERROR_INVALID_VALUE, "alpha/beta pointer is null");
    dgt_status st = validate_gemm(h, transa, transb, m, n, k, A, lda, B, ldb, C, ldc);
    if (st != DGT_SUCCESS) return st;
    if (m == 0 || n == 0) return DGT_SUCCESS;
    if (mode == DGT_FP64_AUTO) {
        if (const TuneEntry* e = tune_lookup(h, DGT_FP64_AUTO, m, n, k)) {
            mode = (dgt_fp64_mode)e->mode;
            slices = e->slices;
        } else {
            mode = DGT_FP64_OZAKI_INT8;
        }
    }
    if (mode != DGT_FP64_NATIVE && !valid_slices(mode, slices))
        return fail(h, DGT_ERROR_INVALID_VALUE, "slice count must be in [2, 16] (moduli: [8, 20])");
    const bool ta = is_trans(transa), tb = is_trans(transb);
    const double a = *alpha, b = *beta;
    const bool read_c = b != 0.0;

    // panel width: about an eighth of n, at least two waves of 128 x 256 output tiles
    int64_t nb = panel_cols;
    if (nb <= 0) {
        const int64_t eighth = ceil_div(ceil_div(n, 8), 256) * 256;
        const int64_t waves = ceil_div(ceil_div(2 * (int64_t)h->num_sms * 128 * 256, std::max<int64_t>(m, 1)), 256) * 256;
        nb = std::max(eighth, waves);
    }
    nb = std::min(nb, n);
    const int64_t panels = ceil_div(n, nb);

    // device copies: op(A) as stored (rowsA x colsA, dense), two op(B) panels, two C panels
    const int64_t rowsA = ta ? k : m, colsA = ta ? m : k;
    const int64_t ldb_d = tb ? nb : std::max<int64_t>(k, 1);  // 'T': panel rows of B (nb x k)
    const size_t a_bytes = up256((size_t)rowsA * colsA * 8), b_bytes = up256((size_t)nb * k * 8),
                 c_bytes = up256((size_t)m * nb * 8);
    void* ws = nullptr;
    if ((st = ensure_workspace(h, a_bytes + 2 * b_bytes + 2 * c_bytes, &ws, 3)) != DGT_SUCCESS) return st;
    if ((st = ensure_copy_streams(h)) != DGT_SUCCESS) return st;
    double* dA = (double*)ws;
    double* dB[2] = {(double*)((char*)ws + a_bytes), (double*)((char*)ws + a_bytes + b_bytes)};
    double* dC[2] = {(double*)((char*)ws + a_bytes + 2 * b_bytes),
                     (double*)((char*)ws + a_bytes + 2 * b_bytes + c_bytes)};
    cudaStream_t s = h->stream, si = h->copy_stream[0], so = h->copy_stream[1];
    cudaEvent_t* ev = h->copy_ev;

    // the CRT mode splits op(A) once (one K-chunk); longer K and other modes run per panel
    const bool crt = mode == DGT_FP64_OZAKI2_INT8 && k > 0 && k <= 65536;
    Oz2Shape sh{};
    Oz2Work w{};
    if (crt) {
        if ((st = ozaki2_shape(h, m, nb, k, slices, sh)) != DGT_SUCCESS) return st;
        void* ows = nullptr;
        if ((st = ensure_workspace(h, ozaki2_carve(sh, nb, sh.n_pad, nullptr).bytes, &ows, 0)) != DGT_SUCCESS)
            return st;
        w = ozaki2_carve(sh, nb, sh.n_pad, ows);
    }

    // copies start after the work already queued on the handle's stream
    JoinCopyStreams join;
    join.s = s;
    join.si = si;
    join.so = so;
    join.ei = ev[EV_JOIN_IN];
    join.eo = ev[EV_JOIN_OUT];
    DGT_CUDA_TRY(h, cudaEventRecord(ev[EV_START], s));
    join.armed = true;
    DGT_CUDA_TRY(h, cudaStreamWaitEvent(si, ev[EV_START], 0));
    DGT_CUDA_TRY(h, cudaStreamWaitEvent(so, ev[EV_START], 0));
    if (k > 0) {
        DGT_CUDA_TRY(h, cudaMemcpy2DAsync(dA, rowsA * 8, A, lda * 8, rowsA * 8, colsA, cudaMemcpyDefault, si));
    }
    DGT_CUDA_TRY(h, cudaEventRecord(ev[EV_A], si));

    auto copy_in = [&](int64_t j) -> dgt_status {
        const int buf = (int)(j & 1);
        const int64_t j0 = j * nb, wj = std::min(nb, n - j0);
        if (j >= 2) {  // the buffers' previous panel has been consumed / written back
            DGT_CUDA_TRY(h, cudaStreamWaitEvent(si, ev[EV_BFREE0 + buf], 0));
            if (read_c) DGT_CUDA_TRY(h, cudaStreamWaitEvent(si, ev[EV_OUT0 + buf], 0));
        }
        if (k > 0) {
            if (tb)  // rows j0 .. j0+wj of B (n x k)
                DGT_CUDA_TRY(h, cudaMemcpy2DAsync(dB[buf], ldb_d * 8, B + j0, ldb * 8, wj * 8, k, cudaMemcpyDefault, si));
            else  // columns j0 .. j0+wj of B (k x n)
                DGT_CUDA_TRY(h, cudaMemcpy2DAsync(dB[buf], ldb_d * 8, B + j0 * ldb, ldb * 8, k * 8, wj,
                                                  cudaMemcpyDefault, si));
        }
        if (read_c)
            DGT_CUDA_TRY(h, cudaMemcpy2DAsync(dC[buf], m * 8, C + j0 * ldc, ldc * 8, m * 8, wj, cudaMemcpyDefault, si));
        DGT_CUDA_TRY(h, cudaEventRecord(ev[EV_IN0 + buf], si));
        return DGT_SUCCESS;
    };

    if ((st = copy_in(0)) != DGT_SUCCESS) return st;
    DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, ev[EV_A], 0));
    if (crt && (st = ozaki2_split(h, s, sh, sh.sa, dA, rowsA, m, sh.m_pad, ta, w.amaxA, w.qnA, w.expA, w.planesA)) != DGT_SUCCESS)
        return st;
    for (int64_t j = 0; j < panels; ++j) {
        const int buf = (int)(j & 1);
        const int64_t j0 = j * nb, wj = std::min(nb, n - j0);
        if (j + 1 < panels && (st = copy_in(j + 1)) != DGT_SUCCESS) return st;
        DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, ev[EV_IN0 + buf], 0));
        if (j >= 2 && !read_c) DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, ev[EV_OUT0 + buf], 0));
        if (crt) {
            const int64_t wpad = ozaki2_n_pad(wj);
            if ((st = ozaki2_split(h, s, sh, sh.sb, dB[buf], ldb_d, wj, wpad, !tb, w.amaxB, w.qnB, w.expB, w.planesB)) != DGT_SUCCESS)
                return st;
            DGT_CUDA_TRY(h, cudaEventRecord(ev[EV_BFREE0 + buf], s));
            if ((st = ozaki2_gemm_crt(h, s, sh, wj, wpad, w.planesA, w.expA, w.planesB, w.expB, w.res, a, b, dC[buf],
                                      m, w.sched)) != DGT_SUCCESS)
                return st;
        } else {
            if ((st = dgt_dgemm_ex(h, transa, transb, m, wj, k, alpha, dA, std::max<int64_t>(rowsA, 1), dB[buf], ldb_d,
                                   beta, dC[buf], m, mode, slices)) != DGT_SUCCESS)
                return st;
            DGT_CUDA_TRY(h, cudaEventRecord(ev[EV_BFREE0 + buf], s));
        }
        DGT_CUDA_TRY(h, cudaEventRecord(ev[EV_C0 + buf], s));
        DGT_CUDA_TRY(h, cudaStreamWaitEvent(so, ev[EV_C0 + buf], 0));
        DGT_CUDA_TRY(h, cudaMemcpy2DAsync(C + j0 * ldc, ldc * 8, dC[buf], m * 8, m * 8, wj, cudaMemcpyDefault, so));
        DGT_CUDA_TRY(h, cudaEventRecord(ev[EV_OUT0 + buf], so));
    }
    // the call is complete on the handle's stream once the last results have reached C
    // (the join at scope exit)
    return DGT_SUCCESS;
}
