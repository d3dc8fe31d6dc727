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
static_assert(EV_COUNT <= 24, "dgt_context::copy_ev holds 24 events");

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
    for (auto& e : h->copy_ev)
        if (!e) DGT_CUDA_TRY(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return DGT_SUCCESS;
}

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

// CRT mode in a 2D block order.  op(A) moves in row panels and op(B) in column panels,
// alternately (A_0, B_0, A_1, B_1, ...); each panel is split into residue planes as soon as it
// arrives, straight into its rows of its operand's planes (one [modulus][rows][k] array per
// operand, so any run of panels is one operand for the GEMM), and the blocks it completes --
// the new row panel times every column panel so far, or every row panel so far times the new
// column panel -- run as ONE residue GEMM and one reconstruction, whose result goes back to
// the host in one strided copy.  The host link's input stream therefore overlaps the
// arithmetic from the second panel on, instead of op(A) crossing whole before the first panel
// computes, and the arithmetic runs in 2 R + 2 Q - 2 launches of full-width GEMMs rather than a
// launch per block.  The FP64 staging buffers and the results are double buffered.  Row
// scaling depends on op(A)'s rows alone and column scaling on op(B)'s columns alone, so every
// block equals the whole-matrix device call's bit for bit.
enum {
    E2_START, E2_AIN0, E2_AIN1, E2_AFREE0, E2_AFREE1, E2_BIN0, E2_BIN1, E2_BFREE0, E2_BFREE1, E2_CIN0, E2_CIN1,
    E2_CREADY0, E2_CREADY1, E2_COUT0, E2_COUT1, E2_JOIN_IN, E2_JOIN_OUT, E2_COUNT
};
static_assert(E2_COUNT <= 24, "dgt_context::copy_ev holds 24 events");

static dgt_status crt_host_2d(dgt_context* h, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                              double beta, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                              int64_t ldc, int nmod, int64_t mb, int64_t nb) {
    const bool read_c = beta != 0.0;
    nb = ozaki2_n_pad(nb);  // column panels of whole 256-wide tiles
    const int64_t R = ceil_div(m, mb), Q = ceil_div(n, nb);
    Oz2Shape shp;  // constants, scales and kernel variant (the same for every panel)
    dgt_status st;
    if ((st = ozaki2_shape(h, m, n, k, nmod, shp)) != DGT_SUCCESS) return st;
    const int64_t m_unit = shp.pair ? 2 * 128 : 128, k_pad = shp.k_pad;
    // op(A)'s planes hold every row panel, [modulus][MS rows][k_pad], row panel i at row i mb;
    // op(B)'s likewise, [modulus][NS rows][k_pad], column panel j at row j nb
    const int64_t MS = ceil_div(m, m_unit) * m_unit, NS = ozaki2_n_pad(n);
    if (mb % m_unit) return fail(h, DGT_ERROR_INVALID_VALUE, "row panels of whole tiles");
    // workspace: both operands' planes, per-row / per-column scale data, the residues and the
    // FP64 result of the largest merged GEMM (a column of row panels, or a row of column panels),
    // the unit counter, two FP64 staging buffers per operand, two result buffers
    auto up = [](size_t x) { return (x + 1023) / 1024 * 1024; };
    const size_t blk = std::max((size_t)MS * nb, (size_t)mb * NS);  // elements of the largest merged result
    const size_t o_pA = 0, o_pB = up((size_t)nmod * MS * k_pad);
    const size_t o_amaxA = o_pB + up((size_t)nmod * NS * k_pad), o_qnA = o_amaxA + up((size_t)m * 8),
                 o_expA = o_qnA + up((size_t)m * 8);
    const size_t o_amaxB = o_expA + up((size_t)m * 4), o_qnB = o_amaxB + up((size_t)n * 8),
                 o_expB = o_qnB + up((size_t)n * 8);
    const size_t o_res = o_expB + up((size_t)n * 4);
    const size_t o_sched = o_res + up((size_t)nmod * blk);
    const size_t stA = up((size_t)mb * k * 8), stB = up((size_t)nb * k * 8), cb = up(blk * 8);
    const size_t o_stA = o_sched + 1024, o_stB = o_stA + 2 * stA, o_cb = o_stB + 2 * stB, total = o_cb + 2 * cb;
    void* ws = nullptr;
    if ((st = ensure_workspace(h, total, &ws, 3)) != DGT_SUCCESS) return st;
    if ((st = ensure_copy_streams(h)) != DGT_SUCCESS) return st;
    char* base = (char*)ws;
    auto* planesA = (int8_t*)(base + o_pA);
    auto* planesB = (int8_t*)(base + o_pB);
    auto* amaxA = (unsigned long long*)(base + o_amaxA);
    auto* qnA = (unsigned long long*)(base + o_qnA);
    auto* expA = (int32_t*)(base + o_expA);
    auto* amaxB = (unsigned long long*)(base + o_amaxB);
    auto* qnB = (unsigned long long*)(base + o_qnB);
    auto* expB = (int32_t*)(base + o_expB);
    auto* res = (uint8_t*)(base + o_res);
    auto* sched = (int32_t*)(base + o_sched);
    double* stageA[2] = {(double*)(base + o_stA), (double*)(base + o_stA + stA)};
    double* stageB[2] = {(double*)(base + o_stB), (double*)(base + o_stB + stB)};
    double* cblk[2] = {(double*)(base + o_cb), (double*)(base + o_cb + cb)};
    cudaStream_t s = h->stream, si = h->copy_stream[0], so = h->copy_stream[1];
    cudaEvent_t* ev = h->copy_ev;

    JoinCopyStreams join;
    join.s = s;
    join.si = si;
    join.so = so;
    join.ei = ev[E2_JOIN_IN];
    join.eo = ev[E2_JOIN_OUT];
    DGT_CUDA_TRY(h, cudaEventRecord(ev[E2_START], s));
    join.armed = true;
    DGT_CUDA_TRY(h, cudaStreamWaitEvent(si, ev[E2_START], 0));
    DGT_CUDA_TRY(h, cudaStreamWaitEvent(so, ev[E2_START], 0));

    // op(A) row panel i: 'N' rows r0.. of the m x k matrix; 'T' columns r0.. of the k x m one
    auto take_a = [&](int64_t i) -> dgt_status {
        const int slot = (int)(i & 1);
        const int64_t r0 = i * mb, mi = std::min(mb, m - r0);
        if (i >= 2) DGT_CUDA_TRY(h, cudaStreamWaitEvent(si, ev[E2_AFREE0 + slot], 0));
        if (ta)
            DGT_CUDA_TRY(h, cudaMemcpy2DAsync(stageA[slot], k * 8, A + r0 * lda, lda * 8, k * 8, mi, cudaMemcpyDefault,
                                              si));
        else
            DGT_CUDA_TRY(h, cudaMemcpy2DAsync(stageA[slot], mi * 8, A + r0, lda * 8, mi * 8, k, cudaMemcpyDefault, si));
        DGT_CUDA_TRY(h, cudaEventRecord(ev[E2_AIN0 + slot], si));
        DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, ev[E2_AIN0 + slot], 0));
        const int64_t pad = std::min(mb, MS - r0);
        if ((st = ozaki2_split(h, s, shp, shp.sa, stageA[slot], ta ? k : mi, mi, pad, ta, amaxA + r0, qnA + r0,
                               expA + r0, planesA + r0 * k_pad, MS)) != DGT_SUCCESS)
            return st;
        DGT_CUDA_TRY(h, cudaEventRecord(ev[E2_AFREE0 + slot], s));
        return DGT_SUCCESS;
    };
    // op(B) column panel j: 'N' columns c0.. of the k x n matrix; 'T' rows c0.. of the n x k one
    auto take_b = [&](int64_t j) -> dgt_status {
        const int slot = (int)(j & 1);
        const int64_t c0 = j * nb, wj = std::min(nb, n - c0);
        if (j >= 2) DGT_CUDA_TRY(h, cudaStreamWaitEvent(si, ev[E2_BFREE0 + slot], 0));
        if (tb)
            DGT_CUDA_TRY(h, cudaMemcpy2DAsync(stageB[slot], wj * 8, B + c0, ldb * 8, wj * 8, k, cudaMemcpyDefault, si));
        else
            DGT_CUDA_TRY(h, cudaMemcpy2DAsync(stageB[slot], k * 8, B + c0 * ldb, ldb * 8, k * 8, wj, cudaMemcpyDefault,
                                              si));
        DGT_CUDA_TRY(h, cudaEventRecord(ev[E2_BIN0 + slot], si));
        DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, ev[E2_BIN0 + slot], 0));
        if ((st = ozaki2_split(h, s, shp, shp.sb, stageB[slot], tb ? wj : k, wj, ozaki2_n_pad(wj), !tb, amaxB + c0,
                               qnB + c0, expB + c0, planesB + c0 * k_pad, NS)) != DGT_SUCCESS)
            return st;
        DGT_CUDA_TRY(h, cudaEventRecord(ev[E2_BFREE0 + slot], s));
        return DGT_SUCCESS;
    };
    // One merged GEMM: C rows [r0, r0 + rows) x columns [c0, c0 + cols), every block of it
    // already split -- the row panels up to ia times a new column panel, or a new row panel
    // times the column panels up to jb -- residue GEMM, reconstruction, result to the host.
    int64_t merged = 0;
    auto compute = [&](int64_t r0, int64_t rows, int64_t c0, int64_t cols) -> dgt_status {
        const int slot = (int)(merged & 1);
        if (merged >= 2) {  // the buffer's previous result has left
            DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, ev[E2_COUT0 + slot], 0));
            if (read_c) DGT_CUDA_TRY(h, cudaStreamWaitEvent(si, ev[E2_COUT0 + slot], 0));
        }
        if (read_c) {
            DGT_CUDA_TRY(h, cudaMemcpy2DAsync(cblk[slot], rows * 8, C + r0 + c0 * ldc, ldc * 8, rows * 8, cols,
                                              cudaMemcpyDefault, si));
            DGT_CUDA_TRY(h, cudaEventRecord(ev[E2_CIN0 + slot], si));
            DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, ev[E2_CIN0 + slot], 0));
        }
        Oz2Shape sh = shp;  // the merged GEMM's rows
        sh.m = rows;
        sh.m_pad = ceil_div(rows, m_unit) * m_unit;
        const int64_t cpad = ozaki2_n_pad(cols);
        if ((st = ozaki2_residue_gemm(h, s, sh, cols, cpad, planesA + r0 * k_pad, planesB + c0 * k_pad, res, sched,
                                      MS, (int64_t)nmod * MS - r0, NS, (int64_t)nmod * NS - c0)) != DGT_SUCCESS)
            return st;
        if ((st = ozaki2_reconstruct(h, s, sh, cols, cpad, res, expA + r0, expB + c0, alpha, beta, cblk[slot],
                                     rows)) != DGT_SUCCESS)
            return st;
        DGT_CUDA_TRY(h, cudaEventRecord(ev[E2_CREADY0 + slot], s));
        DGT_CUDA_TRY(h, cudaStreamWaitEvent(so, ev[E2_CREADY0 + slot], 0));
        DGT_CUDA_TRY(h, cudaMemcpy2DAsync(C + r0 + c0 * ldc, ldc * 8, cblk[slot], rows * 8, rows * 8, cols,
                                          cudaMemcpyDefault, so));
        DGT_CUDA_TRY(h, cudaEventRecord(ev[E2_COUT0 + slot], so));
        ++merged;
        return DGT_SUCCESS;
    };
    // growing rectangle: after each panel, the row or column of blocks it completes, as one GEMM
    int64_t ia = 0, jb = 0;
    while (ia < R || jb < Q) {
        if (ia < R && (ia <= jb || jb >= Q)) {
            if ((st = take_a(ia)) != DGT_SUCCESS) return st;
            if (jb > 0 && (st = compute(ia * mb, std::min(mb, m - ia * mb), 0, std::min(jb * nb, n))) != DGT_SUCCESS)
                return st;
            ++ia;
        } else {
            if ((st = take_b(jb)) != DGT_SUCCESS) return st;
            if (ia > 0 && (st = compute(0, std::min(ia * mb, m), jb * nb, std::min(nb, n - jb * nb))) != DGT_SUCCESS)
                return st;
            ++jb;
        }
    }
    return DGT_SUCCESS;
}

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
    // CRT with a tall op(A) (several row panels of about m/8 rows, at least 1024): 2D block order
    if (mode == DGT_FP64_OZAKI2_INT8 && k > 0 && k <= 65536) {
        const int64_t mb = std::max<int64_t>(1024, ceil_div(ceil_div(m, 8), 256) * 256);
        if (mb < m) return crt_host_2d(h, ta, tb, m, n, k, a, b, A, lda, B, ldb, C, ldc, slices, mb, nb);
    }

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
