// C-ABI entry points of libdgt: handle, validation, and the host side of the step
// schedules (SUMMA panels and 2.5D Cannon rotations become K-segment lists of one
// persistent grouped launch).
#include <cuda_runtime.h>

#include <algorithm>
#include <initializer_list>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dgt_internal.cuh"

namespace dgt {

dgt_status device_table(dgt_context* h, int n, const void* const* parts, const size_t* bytes, void** out,
                        size_t* offsets) {
    uint64_t hash = 1469598103934665603ull;  // FNV-1a over every part
    size_t total = 0;
    for (int i = 0; i < n; ++i) {
        offsets[i] = total;
        total += (bytes[i] + 255) / 256 * 256;
        const unsigned char* b = (const unsigned char*)parts[i];
        for (size_t j = 0; j < bytes[i]; ++j) hash = (hash ^ b[j]) * 1099511628211ull;
        hash = (hash ^ (uint64_t)bytes[i]) * 1099511628211ull;
    }
    ++h->table_clock;
    for (auto& t : h->tables)
        if (t.hash == hash && t.bytes == total) {
            t.last_use = h->table_clock;
            *out = t.ptr;
            return DGT_SUCCESS;
        }
    if ((int)h->tables.size() >= kMaxDeviceTables) {
        size_t lru = 0;
        for (size_t i = 1; i < h->tables.size(); ++i)
            if (h->tables[i].last_use < h->tables[lru].last_use) lru = i;
        DGT_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        cudaFree(h->tables[lru].ptr);
        h->tables.erase(h->tables.begin() + (std::ptrdiff_t)lru);
    }
    void* ptr = nullptr;
    cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(total, 256));
    if (e != cudaSuccess) return cuda_fail(h, e, "device table");
    for (int i = 0; i < n; ++i) {
        e = cudaMemcpyAsync((char*)ptr + offsets[i], parts[i], bytes[i], cudaMemcpyHostToDevice, h->stream);
        if (e != cudaSuccess) {
            cudaFree(ptr);
            return cuda_fail(h, e, "device table upload");
        }
    }
    h->tables.push_back(dgt_context::DevTable{hash, total, ptr, h->table_clock});
    *out = ptr;
    return DGT_SUCCESS;
}

dgt_status ensure_workspace(dgt_context* h, size_t bytes, void** out, int slot) {
    if (slot < 0 || slot > 3) return fail(h, DGT_ERROR_INVALID_VALUE, "bad workspace slot");
    void*& ptr = h->ws[slot];
    size_t& cap = h->ws_bytes[slot];
    if (bytes > cap) {
        if (ptr) {
            cudaStreamSynchronize(h->stream);
            cudaFree(ptr);
            ptr = nullptr;
            cap = 0;
        }
        size_t want = std::max(bytes, (size_t)1 << 20);
        cudaError_t e = cudaMalloc(&ptr, want);
        if (e != cudaSuccess) {
            ptr = nullptr;
            return fail(h, DGT_ERROR_ALLOC, std::string("workspace cudaMalloc: ") + cudaGetErrorString(e));
        }
        cap = want;
    }
    *out = ptr;
    return DGT_SUCCESS;
}

void mark(dgt_context* h, int which) {
    if (!h->profile) return;
    if (!h->ev[which]) cudaEventCreate(&h->ev[which]);
    cudaEventRecord(h->ev[which], h->stream);
    if (which == 0) h->ev_split = true;
}

static int nmod(int a, int b) { return ((a % b) + b) % b; }

// Cannon k-block order for rank (i,j,k).  The reference's skew and rotations
// (src/25DCannon.cpp:303-310, :333-334, :364-365) give t_0 = i + j - k*pc3 and
// t_r = t_{r-1} - r (mod pc); that order is kept when the stacks together visit every
// k-block once, else the shift-by-one order t_r = t_0 - r is used (the fix).
static bool cannon_order(int p, int c, int i, int j, int k, int* out) {
    int pc3 = p / c, pc = p;
    std::vector<int> seen(pc, 0);
    for (int kk = 0; kk < c; ++kk) {
        int t = nmod(i + j - kk * pc3, pc);
        for (int r = 0; r < pc3; ++r) {
            if (r > 0) t = nmod(t - r, pc);
            seen[t]++;
        }
    }
    bool covers = std::all_of(seen.begin(), seen.end(), [](int v) { return v == 1; });
    int t = nmod(i + j - k * pc3, pc);
    for (int r = 0; r < pc3; ++r) {
        if (r > 0) t = covers ? nmod(t - r, pc) : nmod(t - 1, pc);
        out[r] = t;
    }
    return covers;
}

// Emulated-FP64 execution of a step schedule.  CRT residues with steps fused (the default,
// DGT_TUNE_FUSE_STEPS 1): every product is one product over the concatenation of its
// K-segments -- as the native kernel, which keeps one accumulator across the segments -- and
// all products run in one grouped pass.  Otherwise (INT8 slices, steps unfused, or a batch
// the grouped form cannot hold) step t of every product is its t-th segment with K > 0 (the
// reference issues one cublasDgemm per step too); the first step applies the product's beta,
// later steps accumulate, each step splits its own operands (scaled on its own panel: the
// numerics of a per-step local GEMM), and all products' step t run as one grouped pass (the
// products of one step write distinct C); a step the grouped form does not support runs
// product by product.
dgt_status run_problems_emulated(dgt_context* h, const std::vector<Problem>& probs,
                                 const std::vector<KSegment>& segs, dgt_fp64_mode mode, int slices,
                                 bool allow_fused = true) {
    if (!valid_slices(mode, slices))
        return fail(h, DGT_ERROR_INVALID_VALUE, "slice count must be in [2, 16] (moduli: [8, 20])");
    if (mode == DGT_FP64_OZAKI2_INT8 && allow_fused && h->fuse_steps) {
        // CRT, fused: every product is ONE product over the concatenation of its K-segments
        // (rows and columns scaled over the whole K, the residue products summed exactly across
        // steps), all products in one grouped pass
        std::vector<OzProblem> batch;
        bool whole = true;
        for (const Problem& pr : probs) {
            if (pr.m <= 0 || pr.n <= 0) continue;
            int64_t kt = 0;
            for (int s = 0; s < pr.seg_count; ++s) kt += std::max<int64_t>(0, segs[pr.seg_begin + s].k);
            if (kt == 0) {
                whole = false;  // C = beta C: the step-by-step form handles it
                break;
            }
            OzProblem b{pr.transa != 0, pr.transb != 0, pr.m, pr.n, kt, pr.alpha, pr.beta, nullptr, 0, nullptr, 0,
                        pr.C, pr.ldc};
            b.segs = &segs[pr.seg_begin];
            b.nseg = pr.seg_count;
            batch.push_back(b);
        }
        if (whole) {
            dgt_status st = ozaki_dgemm_grouped(h, batch, slices, true);
            if (st != DGT_ERROR_UNSUPPORTED) return st;
        }
    }
    std::vector<std::vector<const KSegment*>> steps(probs.size());
    size_t max_steps = 0;
    for (size_t i = 0; i < probs.size(); ++i) {
        const Problem& pr = probs[i];
        if (pr.m <= 0 || pr.n <= 0) continue;
        for (int s = 0; s < pr.seg_count; ++s)
            if (segs[pr.seg_begin + s].k > 0) steps[i].push_back(&segs[pr.seg_begin + s]);
        max_steps = std::max(max_steps, steps[i].size());
        if (steps[i].empty() && pr.beta != 1.0) {  // no K at all: C = beta * C through the native kernel
            std::vector<Problem> one{pr};
            one[0].alpha = 0.0;
            one[0].seg_begin = 0;
            one[0].seg_count = 1;
            std::vector<KSegment> none{KSegment{nullptr, nullptr, 1, 1, 0}};
            dgt_status st = launch_dmma_grouped(h, one, none);
            if (st != DGT_SUCCESS) return st;
        }
    }
    for (size_t t = 0; t < max_steps; ++t) {
        std::vector<OzProblem> batch;
        for (size_t i = 0; i < probs.size(); ++i) {
            if (t >= steps[i].size()) continue;
            const Problem& pr = probs[i];
            const KSegment& sg = *steps[i][t];
            batch.push_back(OzProblem{pr.transa != 0, pr.transb != 0, pr.m, pr.n, sg.k, pr.alpha,
                                      t == 0 ? pr.beta : 1.0, sg.A, sg.lda, sg.B, sg.ldb, pr.C, pr.ldc});
        }
        if (mode == DGT_FP64_OZAKI_INT8 || mode == DGT_FP64_OZAKI2_INT8) {
            dgt_status st = ozaki_dgemm_grouped(h, batch, slices, mode == DGT_FP64_OZAKI2_INT8);
            if (st != DGT_ERROR_UNSUPPORTED) {
                if (st != DGT_SUCCESS) return st;
                continue;
            }
        }
        for (const OzProblem& b : batch) {
            dgt_status st =
                mode == DGT_FP64_OZAKI2_INT8
                    ? ozaki2_dgemm(h, b.ta, b.tb, b.m, b.n, b.k, b.alpha, b.A, b.lda, b.B, b.ldb, b.beta, b.C, b.ldc,
                                   slices)
                    : ozaki_dgemm(h, b.ta, b.tb, b.m, b.n, b.k, b.alpha, b.A, b.lda, b.B, b.ldb, b.beta, b.C, b.ldc,
                                  mode, slices);
            if (st != DGT_SUCCESS) return st;
        }
    }
    return DGT_SUCCESS;
}

dgt_status validate_gemm(dgt_context* h, char ta, char tb, int64_t m, int64_t n, int64_t k, const void* A,
                         int64_t lda, const void* B, int64_t ldb, const void* C, int64_t ldc) {
    if (!valid_op(ta) || !valid_op(tb)) return fail(h, DGT_ERROR_INVALID_VALUE, "transpose must be N, T or C");
    if (m < 0 || n < 0 || k < 0) return fail(h, DGT_ERROR_INVALID_VALUE, "negative dimension");
    int64_t rowsA = is_trans(ta) ? k : m, rowsB = is_trans(tb) ? n : k;
    if (lda < std::max<int64_t>(1, rowsA)) return fail(h, DGT_ERROR_INVALID_VALUE, "lda < rows of A");
    if (ldb < std::max<int64_t>(1, rowsB)) return fail(h, DGT_ERROR_INVALID_VALUE, "ldb < rows of B");
    if (ldc < std::max<int64_t>(1, m)) return fail(h, DGT_ERROR_INVALID_VALUE, "ldc < m");
    if (m > 0 && n > 0 && !C) return fail(h, DGT_ERROR_INVALID_VALUE, "C is null");
    if (m > 0 && n > 0 && k > 0 && (!A || !B)) return fail(h, DGT_ERROR_INVALID_VALUE, "A or B is null");
    return DGT_SUCCESS;
}

// Problems (one per grouped descriptor) for the grouped entry points; descriptors validated.
dgt_status desc_problems(dgt_context* h, int count, const dgt_gemm_desc* d, std::vector<Problem>& probs,
                                std::vector<KSegment>& segs) {
    if (count < 0 || (count > 0 && !d)) return fail(h, DGT_ERROR_INVALID_VALUE, "bad descriptor array");
    for (int i = 0; i < count; ++i) {
        dgt_status st = validate_gemm(h, d[i].transa, d[i].transb, d[i].m, d[i].n, d[i].k, d[i].A, d[i].lda, d[i].B,
                                      d[i].ldb, d[i].C, d[i].ldc);
        if (st != DGT_SUCCESS) return st;
    }
    for (int i = 0; i < count; ++i) {
        Problem p{};
        p.m = d[i].m;
        p.n = d[i].n;
        p.alpha = d[i].k == 0 ? 0.0 : d[i].alpha;
        p.beta = d[i].beta;
        p.C = d[i].C;
        p.ldc = d[i].ldc;
        p.seg_begin = (int32_t)segs.size();
        p.seg_count = 1;
        p.transa = is_trans(d[i].transa);
        p.transb = is_trans(d[i].transb);
        segs.push_back(KSegment{d[i].A, d[i].B, d[i].lda, d[i].ldb, d[i].k});
        probs.push_back(p);
    }
    return DGT_SUCCESS;
}

}  // namespace dgt

using namespace dgt;

extern "C" {

const char* dgt_status_string(dgt_status s) {
    switch (s) {
        case DGT_SUCCESS: return "DGT_SUCCESS";
        case DGT_ERROR_INVALID_VALUE: return "DGT_ERROR_INVALID_VALUE";
        case DGT_ERROR_UNSUPPORTED: return "DGT_ERROR_UNSUPPORTED";
        case DGT_ERROR_CUDA: return "DGT_ERROR_CUDA";
        case DGT_ERROR_TIMEOUT: return "DGT_ERROR_TIMEOUT";
        case DGT_ERROR_ALLOC: return "DGT_ERROR_ALLOC";
        case DGT_ERROR_NOT_INITIALIZED: return "DGT_ERROR_NOT_INITIALIZED";
    }
    return "DGT_UNKNOWN_STATUS";
}

dgt_status dgt_create(dgt_handle_t* handle) {
    if (!handle) return DGT_ERROR_INVALID_VALUE;
    *handle = nullptr;
    auto* h = new dgt_context;
    cudaError_t e = cudaGetDevice(&h->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    if (e == cudaSuccess) e = cudaMalloc(&h->dev_error, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(h->dev_error, 0, sizeof(unsigned int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (h->dev_error) cudaFree(h->dev_error);
        delete h;
        return DGT_ERROR_CUDA;
    }
    *handle = h;
    return DGT_SUCCESS;
}

dgt_status dgt_destroy(dgt_handle_t h) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    cudaStreamSynchronize(h->stream);
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : h->copy_ev)
        if (e) cudaEventDestroy(e);
    for (auto& cs : h->copy_stream)
        if (cs) cudaStreamDestroy(cs);
    for (auto& e : h->work_ev)
        if (e) cudaEventDestroy(e);
    for (auto& ws : h->work_stream)
        if (ws) cudaStreamDestroy(ws);
    for (void* w : h->ws)
        if (w) cudaFree(w);
    for (auto& t : h->tables) cudaFree(t.ptr);
    if (h->dev_error) cudaFree(h->dev_error);
    delete h;
    return DGT_SUCCESS;
}

dgt_status dgt_set_stream(dgt_handle_t h, dgt_stream_t stream) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    h->stream = (cudaStream_t)stream;
    return DGT_SUCCESS;
}

dgt_status dgt_get_stream(dgt_handle_t h, dgt_stream_t* stream) {
    if (!h || !stream) return DGT_ERROR_NOT_INITIALIZED;
    *stream = (dgt_stream_t)h->stream;
    return DGT_SUCCESS;
}

dgt_status dgt_set_fp64_mode(dgt_handle_t h, dgt_fp64_mode mode, int slices) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (mode < DGT_FP64_NATIVE || mode > DGT_FP64_OZAKI2_INT8)
        return fail(h, DGT_ERROR_INVALID_VALUE, "unknown FP64 mode");
    if (mode != DGT_FP64_NATIVE && mode != DGT_FP64_AUTO && !valid_slices(mode, slices))
        return fail(h, DGT_ERROR_INVALID_VALUE, "slice count must be in [2, 16] (moduli: [8, 20])");
    h->fp64_mode = mode;
    h->slices = slices;
    return DGT_SUCCESS;
}

dgt_status dgt_set_tuning(dgt_handle_t h, dgt_tune_knob knob, int32_t value) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    switch (knob) {
        case DGT_TUNE_DMMA_VARIANT:
            if (value < 0 || value >= dmma_variant_count())
                return fail(h, DGT_ERROR_INVALID_VALUE, "unknown DMMA variant");
            h->dmma_variant = value;
            return DGT_SUCCESS;
        case DGT_TUNE_OZAKI_SLICES:
            if (value < 2 || value > 16) return fail(h, DGT_ERROR_INVALID_VALUE, "slice count must be in [2, 16]");
            h->slices = value;
            return DGT_SUCCESS;
        case DGT_TUNE_PROFILE:
            h->profile = value != 0;
            return DGT_SUCCESS;
        case DGT_TUNE_OZAKI_VARIANT:
            if (value < 0 || value > 7) return fail(h, DGT_ERROR_INVALID_VALUE, "unknown Ozaki kernel variant");
            h->ozaki_variant = value;
            return DGT_SUCCESS;
        case DGT_TUNE_TEST_STALL:
            if (value < 0 || value > 2) return fail(h, DGT_ERROR_INVALID_VALUE, "test stall mode must be 0, 1 or 2");
            h->test_stall = value;
            return DGT_SUCCESS;
        case DGT_TUNE_FUSE_STEPS:
            h->fuse_steps = value != 0;
            return DGT_SUCCESS;
        case DGT_TUNE_CRT_PANELS:
            if (value < 0 || value > 8) return fail(h, DGT_ERROR_INVALID_VALUE, "CRT panel count must be in [0, 8]");
            h->crt_panels = value;
            return DGT_SUCCESS;
    }
    return fail(h, DGT_ERROR_INVALID_VALUE, "unknown tuning knob");
}

int32_t dgt_last_timings(dgt_handle_t h, float* out, int32_t n) {
    if (!h || !out || n <= 0 || !h->profile || !h->ev[1] || !h->ev[2]) return 0;
    if (cudaEventSynchronize(h->ev[2]) != cudaSuccess) return 0;
    float split = 0.f, gemm = 0.f;
    if (h->ev_split && h->ev[0]) cudaEventElapsedTime(&split, h->ev[0], h->ev[1]);
    cudaEventElapsedTime(&gemm, h->ev[1], h->ev[2]);
    out[0] = split;
    if (n > 1) out[1] = gemm;
    return n > 1 ? 2 : 1;
}

dgt_status dgt_get_tuning(dgt_handle_t h, dgt_tune_knob knob, int32_t* value) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (!value) return fail(h, DGT_ERROR_INVALID_VALUE, "null output");
    switch (knob) {
        case DGT_TUNE_DMMA_VARIANT: *value = h->dmma_variant; return DGT_SUCCESS;
        case DGT_TUNE_OZAKI_SLICES: *value = h->slices; return DGT_SUCCESS;
        case DGT_TUNE_PROFILE: *value = h->profile ? 1 : 0; return DGT_SUCCESS;
        case DGT_TUNE_OZAKI_VARIANT: *value = h->ozaki_variant; return DGT_SUCCESS;
        case DGT_TUNE_TEST_STALL: *value = h->test_stall; return DGT_SUCCESS;
        case DGT_TUNE_FUSE_STEPS: *value = h->fuse_steps ? 1 : 0; return DGT_SUCCESS;
        case DGT_TUNE_CRT_PANELS: *value = h->crt_panels; return DGT_SUCCESS;
    }
    return fail(h, DGT_ERROR_INVALID_VALUE, "unknown tuning knob");
}

const char* dgt_last_error(dgt_handle_t h) { return h ? h->last_error.c_str() : "null handle"; }

dgt_status dgt_check_device(dgt_handle_t h) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    DGT_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    unsigned int word = 0;
    DGT_CUDA_TRY(h, cudaMemcpy(&word, h->dev_error, sizeof(word), cudaMemcpyDeviceToHost));
    DGT_CUDA_TRY(h, cudaMemset(h->dev_error, 0, sizeof(word)));
    if (word & DGT_DEVERR_TIMEOUT) return fail(h, DGT_ERROR_TIMEOUT, "a device-side wait exceeded its budget");
    if (word & DGT_DEVERR_BOUNDS) return fail(h, DGT_ERROR_INVALID_VALUE, "a device-side bounds check failed");
    return DGT_SUCCESS;
}

int64_t dgt_launch_count(dgt_handle_t h) { return h ? h->launches.load() : 0; }

int32_t dgt_numroc(int32_t n, int32_t nb, int32_t iproc, int32_t isrproc, int32_t nprocs) {
    // pblasDecomposition.cpp:3-23
    if (nb <= 0 || nprocs <= 0) return 0;
    int myDistance = (nprocs + iproc - isrproc) % nprocs;
    int numBlocks = n / nb;
    int r = (numBlocks / nprocs) * nb;
    int extra = numBlocks % nprocs;
    if (myDistance < extra)
        r += nb;
    else if (myDistance == extra)
        r += n % nb;
    return r;
}

dgt_status dgt_block2d_grid(int32_t P, int32_t* dRow, int32_t* dCol) {
    // calculateVirtualDeviceGrid, 2DBlockSequentialDecomposition.cpp:27-54
    if (P <= 0 || !dRow || !dCol) return DGT_ERROR_INVALID_VALUE;
    int Px = (int)std::sqrt((double)P), Py = Px;
    if (Px == 0) {
        Py = P;
        Px = 1;
    }
    int counter;
    for (counter = Px; counter > 0; --counter)
        if (P % counter == 0) break;
    if (counter == 0) {
        Px = P;
        Py = 1;
    } else {
        Px = counter;
        Py = P / counter;
    }
    *dRow = Py;
    *dCol = Px;
    return DGT_SUCCESS;
}

int32_t dgt_cannon_schedule(int32_t p, int32_t c, int32_t i, int32_t j, int32_t k, int32_t* out) {
    if (p <= 0 || c <= 0 || p % c != 0 || !out) return -1;
    return cannon_order(p, c, i, j, k, out) ? 1 : 0;
}

// ---- local GEMM -----------------------------------------------------------------------


static dgt_status native_single(dgt_context* h, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                                const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                                int64_t ldc) {
    std::vector<Problem> probs(1);
    Problem& p = probs[0];
    p.m = m;
    p.n = n;
    p.alpha = (k == 0) ? 0.0 : alpha;
    p.beta = beta;
    p.C = C;
    p.ldc = ldc;
    p.seg_begin = 0;
    p.seg_count = 1;
    p.transa = is_trans(ta);
    p.transb = is_trans(tb);
    std::vector<KSegment> segs{KSegment{A, B, lda, ldb, k}};
    h->ev_split = false;
    mark(h, 1);
    dgt_status st = launch_dmma_grouped(h, probs, segs);
    mark(h, 2);
    return st;
}

dgt_status dgt_dgemm_ex(dgt_handle_t h, char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha,
                        const double* A, int64_t lda, const double* B, int64_t ldb, const double* beta, double* C,
                        int64_t ldc, dgt_fp64_mode mode, int slices) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (!alpha || !beta) return fail(h, DGT_ERROR_INVALID_VALUE, "alpha/beta pointer is null");
    dgt_status st = validate_gemm(h, ta, tb, m, n, k, A, lda, B, ldb, C, ldc);
    if (st != DGT_SUCCESS) return st;
    if (m == 0 || n == 0) return DGT_SUCCESS;
    // tuned choices for this shape class, if the autotuner has seen one
    int dv = h->dmma_variant, ov = h->ozaki_variant;
    if (mode == DGT_FP64_AUTO) {
        const TuneEntry* e = tune_lookup(h, DGT_FP64_AUTO, m, n, k);
        if (e) {
            mode = (dgt_fp64_mode)e->mode;
            slices = e->slices;
            (e->mode == DGT_FP64_NATIVE ? dv : ov) = e->variant;
        } else {
            mode = DGT_FP64_OZAKI_INT8;
        }
    }
    if (const TuneEntry* e = tune_lookup(h, mode, m, n, k)) (mode == DGT_FP64_NATIVE ? dv : ov) = e->variant;
    struct Restore {
        dgt_context* h;
        int dv, ov;
        ~Restore() {
            h->dmma_variant = dv;
            h->ozaki_variant = ov;
        }
    } restore{h, h->dmma_variant, h->ozaki_variant};
    h->dmma_variant = dv;
    h->ozaki_variant = ov;
    if (mode == DGT_FP64_NATIVE || k == 0)
        return native_single(h, ta, tb, m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc);
    if (!valid_slices(mode, slices))
        return fail(h, DGT_ERROR_INVALID_VALUE, "slice count must be in [2, 16] (moduli: [8, 20])");
    if (mode == DGT_FP64_OZAKI2_INT8)
        return ozaki2_dgemm(h, is_trans(ta), is_trans(tb), m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc, slices);
    return ozaki_dgemm(h, is_trans(ta), is_trans(tb), m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc, mode, slices);
}

dgt_status dgt_dgemm_workspace_size(int64_t m, int64_t n, int64_t k, dgt_fp64_mode mode, int slices,
                                    size_t* bytes) {
    if (!bytes) return DGT_ERROR_INVALID_VALUE;
    *bytes = 0;
    if (m < 0 || n < 0 || k < 0) return DGT_ERROR_INVALID_VALUE;
    if (m == 0 || n == 0 || k == 0 || mode == DGT_FP64_NATIVE) return DGT_SUCCESS;
    if (mode == DGT_FP64_OZAKI_INT8 || mode == DGT_FP64_OZAKI_BF16) {
        if (!valid_slices(mode, slices)) return DGT_ERROR_INVALID_VALUE;
        return ozaki_workspace_bound(slices, m, n, k, mode == DGT_FP64_OZAKI_BF16, bytes);
    }
    if (mode == DGT_FP64_OZAKI2_INT8) {
        if (!valid_slices(mode, slices)) return DGT_ERROR_INVALID_VALUE;
        return ozaki2_workspace_bound(slices, m, n, k, bytes);
    }
    if (mode == DGT_FP64_AUTO) {  // the autotuner's emulated candidates for this count
        size_t a = 0, c = 0;
        dgt_status sa = valid_slices(DGT_FP64_OZAKI_INT8, slices)
                            ? ozaki_workspace_bound(slices, m, n, k, false, &a) : DGT_ERROR_INVALID_VALUE;
        dgt_status sc = ozaki2_workspace_bound(valid_slices(DGT_FP64_OZAKI2_INT8, slices) ? slices : 16, m, n, k, &c);
        if (sa != DGT_SUCCESS && sc != DGT_SUCCESS) return sa;
        *bytes = std::max(a, c);
        return DGT_SUCCESS;
    }
    return DGT_ERROR_INVALID_VALUE;
}

dgt_status dgt_dgemm(dgt_handle_t h, char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha,
                     const double* A, int64_t lda, const double* B, int64_t ldb, const double* beta, double* C,
                     int64_t ldc) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    return dgt_dgemm_ex(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, h->fp64_mode, h->slices);
}

dgt_status dgt_dgemm_grouped(dgt_handle_t h, int count, const dgt_gemm_desc* d, dgt_fp64_mode mode, int slices) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    std::vector<Problem> probs;
    std::vector<KSegment> segs;
    probs.reserve(count > 0 ? count : 0);
    segs.reserve(count > 0 ? count : 0);
    dgt_status st = desc_problems(h, count, d, probs, segs);
    if (st != DGT_SUCCESS) return st;
    if (mode == DGT_FP64_AUTO) mode = DGT_FP64_NATIVE;
    if (mode != DGT_FP64_NATIVE) return run_problems_emulated(h, probs, segs, mode, slices);
    return launch_dmma_grouped(h, probs, segs);
}

// ---- SUMMA on block-cyclic local buffers -------------------------------------------------

// Shape checks of a SUMMA call (dgt_summa, dgt_summa_rank, dgt_summa_schedule); nullptr if
// the call is valid, else the reason.  lldC, when given, is checked for every rank.
static const char* summa_check(const dgt_grid_layout* L, int64_t M, int64_t N, int64_t K, const int64_t* lldA,
                               const int64_t* lldB, const int64_t* lldC) {
    const int p = L->p, q = L->q;
    if (p <= 0 || q <= 0 || L->c != 1) return "SUMMA needs p, q >= 1 and c == 1";
    if (L->mb <= 0 || L->nb <= 0 || L->kb <= 0) return "block sizes must be > 0";
    if (M < 0 || N < 0 || K < 0 || M > INT32_MAX || N > INT32_MAX || K > INT32_MAX) return "dimension out of range";
    auto roc = [](int64_t n, int64_t b, int i, int np) { return (int64_t)dgt_numroc((int)n, (int)b, i, 0, np); };
    for (int r = 0; r < p * q; ++r) {
        int i = r / q;
        if (lldC && lldC[r] < std::max<int64_t>(1, roc(M, L->mb, i, p))) return "lldC < rows";
        if (lldA[r] < std::max<int64_t>(1, roc(M, L->mb, i, p))) return "lldA < rows";
        if (lldB[r] < std::max<int64_t>(1, roc(K, L->kb, i, p))) return "lldB < rows";
    }
    return nullptr;
}

// Virtual rank (i, j)'s SUMMA problem: its C block and the K segments its GEMM walks.  Panel
// t reads A's block column t from process column t mod q (local column (t div q) kb) and
// B's block row t from process row t mod p (local row (t div p) kb), through A_loc / B_loc,
// which may point into other devices' memory.  Panels are visited owner pair by owner pair
// (t mod q, t mod p) so that runs contiguous in both owners' buffers merge into one segment.
static Problem summa_problem(const dgt_grid_layout* L, int i, int j, int64_t M, int64_t N, int64_t K, double alpha,
                             double beta, const double* const* A_loc, const int64_t* lldA,
                             const double* const* B_loc, const int64_t* lldB, double* C, int64_t ldc,
                             std::vector<KSegment>& segs) {
    const int p = L->p, q = L->q;
    const int64_t mb = L->mb, nb = L->nb, kb = L->kb;
    auto roc = [](int64_t n, int64_t b, int i, int np) { return (int64_t)dgt_numroc((int)n, (int)b, i, 0, np); };
    const int64_t kblocks = ceil_div(K, kb);
    Problem pr{};
    pr.m = roc(M, mb, i, p);
    pr.n = roc(N, nb, j, q);
    pr.alpha = K == 0 ? 0.0 : alpha;
    pr.beta = beta;
    pr.C = C;
    pr.ldc = ldc;
    pr.seg_begin = (int32_t)segs.size();
    std::vector<std::vector<int64_t>> classes;
    std::vector<std::pair<int, int>> keys;
    for (int64_t t = 0; t < kblocks; ++t) {
        std::pair<int, int> key((int)(t % q), (int)(t % p));
        auto it = std::find(keys.begin(), keys.end(), key);
        if (it == keys.end()) {
            keys.push_back(key);
            classes.push_back({t});
        } else {
            classes[it - keys.begin()].push_back(t);
        }
    }
    for (auto& cls : classes) {
        for (int64_t t : cls) {
            int ra = i * q + (int)(t % q);
            int rb = (int)(t % p) * q + j;
            int64_t kt = std::min(kb, K - t * kb);
            const double* a = A_loc[ra] + (t / q) * kb * lldA[ra];
            const double* b = B_loc[rb] + (t / p) * kb;
            if (pr.seg_count > 0) {
                KSegment& last = segs.back();
                if (last.lda == lldA[ra] && last.ldb == lldB[rb] && last.A + last.k * last.lda == a &&
                    last.B + last.k == b) {
                    last.k += kt;
                    continue;
                }
            }
            segs.push_back(KSegment{a, b, lldA[ra], lldB[rb], kt});
            pr.seg_count++;
        }
    }
    if (pr.seg_count == 0) {  // K == 0: C = beta*C
        segs.push_back(KSegment{nullptr, nullptr, 1, 1, 0});
        pr.seg_count = 1;
    }
    return pr;
}

dgt_status dgt_summa(dgt_handle_t h, const dgt_grid_layout* L, int64_t M, int64_t N, int64_t K, double alpha,
                     const double* const* A_loc, const int64_t* lldA, const double* const* B_loc,
                     const int64_t* lldB, double beta, double* const* C_loc, const int64_t* lldC, dgt_fp64_mode mode,
                     int slices) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (!L || !A_loc || !B_loc || !C_loc || !lldA || !lldB || !lldC)
        return fail(h, DGT_ERROR_INVALID_VALUE, "null argument");
    if (const char* why = summa_check(L, M, N, K, lldA, lldB, lldC)) return fail(h, DGT_ERROR_INVALID_VALUE, why);
    if (mode == DGT_FP64_AUTO) mode = DGT_FP64_NATIVE;
    std::vector<Problem> probs;
    std::vector<KSegment> segs;
    for (int i = 0; i < L->p; ++i)
        for (int j = 0; j < L->q; ++j) {
            const int r = i * L->q + j;
            probs.push_back(summa_problem(L, i, j, M, N, K, alpha, beta, A_loc, lldA, B_loc, lldB, C_loc[r], lldC[r],
                                          segs));
        }
    if (mode == DGT_FP64_NATIVE) return launch_dmma_grouped(h, probs, segs);
    return run_problems_emulated(h, probs, segs, mode, slices);
}

dgt_status dgt_summa_rank(dgt_handle_t h, const dgt_grid_layout* L, int32_t rank, int64_t M, int64_t N, int64_t K,
                          double alpha, const double* const* A_loc, const int64_t* lldA, const double* const* B_loc,
                          const int64_t* lldB, double beta, double* C, int64_t ldc, dgt_fp64_mode mode, int slices) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (!L || !A_loc || !B_loc || !C || !lldA || !lldB) return fail(h, DGT_ERROR_INVALID_VALUE, "null argument");
    if (const char* why = summa_check(L, M, N, K, lldA, lldB, nullptr)) return fail(h, DGT_ERROR_INVALID_VALUE, why);
    if (rank < 0 || rank >= L->p * L->q) return fail(h, DGT_ERROR_INVALID_VALUE, "rank outside the grid");
    const int i = rank / L->q, j = rank % L->q;
    if (ldc < std::max<int64_t>(1, dgt_numroc((int)M, (int)L->mb, i, 0, L->p)))
        return fail(h, DGT_ERROR_INVALID_VALUE, "ldc < rows");
    if (mode == DGT_FP64_AUTO) mode = DGT_FP64_NATIVE;
    std::vector<KSegment> segs;
    std::vector<Problem> probs{summa_problem(L, i, j, M, N, K, alpha, beta, A_loc, lldA, B_loc, lldB, C, ldc, segs)};
    if (probs[0].m == 0 || probs[0].n == 0) return DGT_SUCCESS;
    if (mode == DGT_FP64_NATIVE) return launch_dmma_grouped(h, probs, segs);
    return run_problems_emulated(h, probs, segs, mode, slices);
}

int32_t dgt_summa_schedule(const dgt_grid_layout* L, int32_t rank, int64_t M, int64_t N, int64_t K,
                           const double* const* A_loc, const int64_t* lldA, const double* const* B_loc,
                           const int64_t* lldB, int64_t* out, int32_t max_segments) {
    if (!L || !A_loc || !B_loc || !lldA || !lldB || summa_check(L, M, N, K, lldA, lldB, nullptr)) return -1;
    if (rank < 0 || rank >= L->p * L->q) return -1;
    std::vector<KSegment> segs;
    double* no_c = nullptr;
    summa_problem(L, rank / L->q, rank % L->q, M, N, K, 1.0, 0.0, A_loc, lldA, B_loc, lldB, no_c, 1, segs);
    for (size_t s = 0; s < segs.size() && out && (int32_t)s < max_segments; ++s) {
        out[5 * s + 0] = (int64_t)(uintptr_t)segs[s].A;
        out[5 * s + 1] = (int64_t)(uintptr_t)segs[s].B;
        out[5 * s + 2] = segs[s].lda;
        out[5 * s + 3] = segs[s].ldb;
        out[5 * s + 4] = segs[s].k;
    }
    return (int32_t)segs.size();
}

// ---- buffers shared between processes (CUDA IPC) --------------------------------------------

static_assert(sizeof(dgt_ipc_handle) == sizeof(cudaIpcMemHandle_t), "IPC handle size");

dgt_status dgt_ipc_alloc(size_t bytes, void** ptr, dgt_ipc_handle* handle) {
    if (!ptr || !handle || bytes == 0) return DGT_ERROR_INVALID_VALUE;
    *ptr = nullptr;
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return DGT_ERROR_ALLOC;
    }
    cudaIpcMemHandle_t h;
    if (cudaIpcGetMemHandle(&h, p) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return DGT_ERROR_CUDA;
    }
    std::memcpy(handle->bytes, &h, sizeof(h));
    *ptr = p;
    return DGT_SUCCESS;
}

dgt_status dgt_ipc_open(const dgt_ipc_handle* handle, void** ptr) {
    if (!ptr || !handle) return DGT_ERROR_INVALID_VALUE;
    *ptr = nullptr;
    cudaIpcMemHandle_t h;
    std::memcpy(&h, handle->bytes, sizeof(h));
    if (cudaIpcOpenMemHandle(ptr, h, cudaIpcMemLazyEnablePeerAccess) != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return DGT_ERROR_CUDA;
    }
    return DGT_SUCCESS;
}

dgt_status dgt_ipc_close(void* ptr) {
    if (!ptr) return DGT_ERROR_INVALID_VALUE;
    if (cudaIpcCloseMemHandle(ptr) != cudaSuccess) {
        cudaGetLastError();
        return DGT_ERROR_CUDA;
    }
    return DGT_SUCCESS;
}

dgt_status dgt_ipc_free(void* ptr) {
    if (!ptr) return DGT_ERROR_INVALID_VALUE;
    if (cudaFree(ptr) != cudaSuccess) {
        cudaGetLastError();
        return DGT_ERROR_CUDA;
    }
    return DGT_SUCCESS;
}

// ---- 2.5D Cannon -----------------------------------------------------------------------------

dgt_status dgt_cannon25d(dgt_handle_t h, int64_t M, int32_t p, int32_t c, char ta, char tb, double alpha,
                         const double* const* A_tiles, const double* const* B_tiles, double beta,
                         double* const* C_tiles, dgt_fp64_mode mode, int slices) {
    return dgt_cannon25d_batch(h, M, p, c, ta, tb, alpha, A_tiles, B_tiles, beta, C_tiles, 0, nullptr, mode, slices);
}

dgt_status dgt_cannon25d_batch(dgt_handle_t h, int64_t M, int32_t p, int32_t c, char ta, char tb, double alpha,
                               const double* const* A_tiles, const double* const* B_tiles, double beta,
                               double* const* C_tiles, int32_t count, const dgt_gemm_desc* descs,
                               dgt_fp64_mode mode, int slices) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (!A_tiles || !B_tiles || !C_tiles) return fail(h, DGT_ERROR_INVALID_VALUE, "null tile array");
    // Summa25Decomposer ctor checks (src/25DCannon.cpp:7-23), as status codes
    if (p <= 0 || c <= 0 || p % c != 0) return fail(h, DGT_ERROR_INVALID_VALUE, "need p % c == 0");
    if (M <= 0 || M % p != 0) return fail(h, DGT_ERROR_INVALID_VALUE, "need M % p == 0");
    if (!valid_op(ta) || !valid_op(tb)) return fail(h, DGT_ERROR_INVALID_VALUE, "transpose must be N, T or C");
    if (p * p > 256) return fail(h, DGT_ERROR_UNSUPPORTED, "more than 256 tiles per stack");
    if (mode == DGT_FP64_AUTO) mode = DGT_FP64_NATIVE;
    if (mode != DGT_FP64_NATIVE && !valid_slices(mode, slices))
        return fail(h, DGT_ERROR_INVALID_VALUE, "slice count must be in [2, 16] (moduli: [8, 20])");
    std::vector<Problem> extra;
    std::vector<KSegment> extra_segs;
    dgt_status st = desc_problems(h, count, descs, extra, extra_segs);
    if (st != DGT_SUCCESS) return st;
    const int64_t lm = M / p, tile = lm * lm;
    const int pc3 = p / c;
    const bool native = mode == DGT_FP64_NATIVE;
    const bool fuse = h->fuse_steps && (native ? (c > 1 || count > 0) : mode == DGT_FP64_OZAKI2_INT8);
    // native stacks 1..c-1 write partial tiles W; fused, the stack-0 tiles wait on counters
    // after W for them
    const int64_t tiles_per = native ? dmma_tile_count(lm, lm) : 0;
    double* W = nullptr;
    int32_t* flags = nullptr;
    const size_t w_bytes = (size_t)(c - 1) * p * p * tile * sizeof(double);
    const size_t flag_count = (size_t)p * p * tiles_per;
    if (c > 1 && (native || !fuse)) {
        void* ws = nullptr;
        st = ensure_workspace(h, w_bytes + (fuse ? flag_count * sizeof(int32_t) : 0), &ws, 2);
        if (st != DGT_SUCCESS) return st;
        W = (double*)ws;
        flags = fuse ? (int32_t*)((char*)ws + w_bytes) : nullptr;
    }
    // every virtual rank (i, j, k): one problem whose K-segments are its k-blocks in Cannon
    // order; stack 0 carries beta*C (src/25DCannon.cpp:322), the other stacks start at 0
    std::vector<int> order(pc3);
    auto rank_problem = [&](int i, int j, int k, std::vector<Problem>& probs, std::vector<KSegment>& segs) {
        cannon_order(p, c, i, j, k, order.data());
        Problem pr{};
        pr.m = lm;
        pr.n = lm;
        pr.alpha = alpha;
        pr.beta = (k == 0) ? beta : 0.0;
        pr.C = (k == 0 || !W) ? C_tiles[i * p + j] : W + ((int64_t)(k - 1) * p * p + i * p + j) * tile;
        pr.ldc = lm;
        pr.transa = is_trans(ta);
        pr.transb = is_trans(tb);
        pr.seg_begin = (int32_t)segs.size();
        pr.seg_count = pc3;
        for (int s = 0; s < pc3; ++s) {
            const int t = order[s];
            segs.push_back(KSegment{A_tiles[i * p + t], B_tiles[t * p + j], lm, lm, lm});
        }
        probs.push_back(pr);
    };
    std::vector<Problem> probs;
    std::vector<KSegment> segs;
    if (fuse && native) {
        // ONE persistent launch: every partial tile first (they only store and count
        // themselves), then the extra products, then the stack-0 tiles, which add their
        // partials in stack order once counted (reduceResult, src/25DCannon.cpp:203-228)
        for (int k = 1; k < c; ++k)
            for (int i = 0; i < p; ++i)
                for (int j = 0; j < p; ++j) {
                    rank_problem(i, j, k, probs, segs);
                    probs.back().red_role = 1;
                    probs.back().red_slot = (int32_t)((i * p + j) * tiles_per);
                }
        for (Problem e : extra) {
            e.seg_begin += (int32_t)segs.size();
            probs.push_back(e);
        }
        segs.insert(segs.end(), extra_segs.begin(), extra_segs.end());
        // rank_problem's segments go after the extras' (seg_begin is taken at the push)
        for (int i = 0; i < p; ++i)
            for (int j = 0; j < p; ++j) {
                rank_problem(i, j, 0, probs, segs);
                if (c == 1) continue;
                Problem& pr = probs.back();
                pr.red_role = 2;
                pr.red_slot = (int32_t)((i * p + j) * tiles_per);
                pr.red_wait = c - 1;
                pr.red_src = W + (int64_t)(i * p + j) * tile;
                pr.red_stride = (int64_t)p * p * tile;
                pr.red_ld = lm;
            }
        return launch_dmma_grouped(h, probs, segs, flags, flag_count);
    }
    if (fuse) {
        // CRT: one grouped pass; each (i, j) is a stack group -- stack 0's product, then stacks
        // 1..c-1 as further stacks of the same output -- and every rank's k-blocks are one K
        for (int i = 0; i < p; ++i)
            for (int j = 0; j < p; ++j)
                for (int k = 0; k < c; ++k) rank_problem(i, j, k, probs, segs);
        const size_t cannon_probs = probs.size();
        for (Problem e : extra) {
            e.seg_begin += (int32_t)segs.size();
            probs.push_back(e);
        }
        segs.insert(segs.end(), extra_segs.begin(), extra_segs.end());
        std::vector<OzProblem> batch;
        for (size_t r = 0; r < probs.size(); ++r) {
            const Problem& pr = probs[r];
            if (pr.m <= 0 || pr.n <= 0) continue;
            int64_t kt = 0;
            for (int s = 0; s < pr.seg_count; ++s) kt += segs[pr.seg_begin + s].k;
            if (kt == 0) {  // an extra product without K: C = beta C (the native kernel, alpha 0)
                std::vector<Problem> one{pr};
                std::vector<KSegment> none{KSegment{nullptr, nullptr, 1, 1, 0}};
                one[0].seg_begin = 0;
                st = launch_dmma_grouped(h, one, none);
                if (st != DGT_SUCCESS) return st;
                continue;
            }
            OzProblem b{pr.transa != 0, pr.transb != 0, pr.m, pr.n, kt, pr.alpha, pr.beta, nullptr, 0, nullptr, 0,
                        pr.C, pr.ldc};
            b.segs = &segs[pr.seg_begin];
            b.nseg = pr.seg_count;
            b.stack = (r < cannon_probs && r % c != 0) ? 1 : 0;
            batch.push_back(b);
        }
        st = ozaki_dgemm_grouped(h, batch, slices, true);
        if (st != DGT_ERROR_UNSUPPORTED) return st;
        // too large for one pass: the step-by-step form below
        probs.clear();
        segs.clear();
        if (c > 1) {
            void* ws = nullptr;
            st = ensure_workspace(h, w_bytes, &ws, 2);
            if (st != DGT_SUCCESS) return st;
            W = (double*)ws;
        }
    }
    // step-by-step form: the virtual ranks in one grouped call, then the stack reduction, then
    // the extra products as a second grouped call
    for (int k = 0; k < c; ++k)
        for (int i = 0; i < p; ++i)
            for (int j = 0; j < p; ++j) rank_problem(i, j, k, probs, segs);
    st = native ? launch_dmma_grouped(h, probs, segs) : run_problems_emulated(h, probs, segs, mode, slices, false);
    if (st != DGT_SUCCESS) return st;
    // stack reduction (reduceResult, src/25DCannon.cpp:203-228) into the stack-0 tiles
    if (c > 1) {
        st = launch_stack_reduce(h, tile, p * p, c - 1, C_tiles, W, (int64_t)p * p * tile);
        if (st != DGT_SUCCESS) return st;
    }
    if (extra.empty()) return DGT_SUCCESS;
    return native ? launch_dmma_grouped(h, extra, extra_segs) : run_problems_emulated(h, extra, extra_segs, mode, slices);
}

dgt_status dgt_cannon25d_rank(dgt_handle_t h, int64_t M, int32_t p, int32_t c, int32_t rank, char ta, char tb,
                              double alpha, const double* const* A_tiles, const double* const* B_tiles, double beta,
                              double* C_tile, dgt_fp64_mode mode, int slices) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (!A_tiles || !B_tiles || !C_tile) return fail(h, DGT_ERROR_INVALID_VALUE, "null tile array or C tile");
    if (p <= 0 || c <= 0 || p % c != 0) return fail(h, DGT_ERROR_INVALID_VALUE, "need p % c == 0");
    if (M <= 0 || M % p != 0) return fail(h, DGT_ERROR_INVALID_VALUE, "need M % p == 0");
    if (!valid_op(ta) || !valid_op(tb)) return fail(h, DGT_ERROR_INVALID_VALUE, "transpose must be N, T or C");
    if (rank < 0 || rank >= p * p * c) return fail(h, DGT_ERROR_INVALID_VALUE, "rank outside the grid");
    if (mode == DGT_FP64_AUTO) mode = DGT_FP64_NATIVE;
    const int64_t lm = M / p;
    const int pc3 = p / c;
    const int k = rank / (p * p), i = (rank / p) % p, j = rank % p;
    std::vector<int> order(pc3);
    cannon_order(p, c, i, j, k, order.data());
    Problem pr{};
    pr.m = lm;
    pr.n = lm;
    pr.alpha = alpha;
    pr.beta = (k == 0) ? beta : 0.0;  // the other stacks' partial sums start at 0
    pr.C = C_tile;
    pr.ldc = lm;
    pr.transa = is_trans(ta);
    pr.transb = is_trans(tb);
    pr.seg_begin = 0;
    pr.seg_count = pc3;
    std::vector<KSegment> segs;
    for (int s = 0; s < pc3; ++s) {
        int t = order[s];
        segs.push_back(KSegment{A_tiles[i * p + t], B_tiles[t * p + j], lm, lm, lm});
    }
    std::vector<Problem> probs{pr};
    return (mode == DGT_FP64_NATIVE) ? launch_dmma_grouped(h, probs, segs)
                                     : run_problems_emulated(h, probs, segs, mode, slices);
}

dgt_status dgt_reduce_tiles(dgt_handle_t h, double* C, const double* const* parts, int32_t nparts, int64_t elems) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (elems < 0 || nparts < 0) return fail(h, DGT_ERROR_INVALID_VALUE, "negative size");
    if (elems == 0 || nparts == 0) return DGT_SUCCESS;
    if (!C || !parts) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    for (int s = 0; s < nparts; ++s)
        if (!parts[s]) return fail(h, DGT_ERROR_INVALID_VALUE, "null part");
    return launch_tile_sum(h, C, parts, nparts, elems);
}

// ---- layout ------------------------------------------------------------------------------------

static dgt_status check_cyclic(dgt_context* h, int64_t M, int64_t N, int64_t mb, int64_t nb, int p, int q,
                               const void* g, int64_t ldg, const void* locals, const int64_t* lld) {
    if (M < 0 || N < 0 || mb <= 0 || nb <= 0 || p <= 0 || q <= 0)
        return fail(h, DGT_ERROR_INVALID_VALUE, "bad sizes or grid");
    if (M > INT32_MAX || N > INT32_MAX) return fail(h, DGT_ERROR_INVALID_VALUE, "dimension out of range");
    if (ldg < std::max<int64_t>(1, M)) return fail(h, DGT_ERROR_INVALID_VALUE, "ldg < M");
    if (!g || !locals || !lld) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    for (int r = 0; r < p * q; ++r) {
        int64_t rows = dgt_numroc((int)M, (int)mb, r / q, 0, p);
        if (lld[r] < std::max<int64_t>(1, rows)) return fail(h, DGT_ERROR_INVALID_VALUE, "lld < local rows");
    }
    return DGT_SUCCESS;
}

dgt_status dgt_pack_block_cyclic(dgt_handle_t h, int64_t M, int64_t N, int64_t mb, int64_t nb, int32_t p, int32_t q,
                                 const double* global, int64_t ldg, double* const* locals, const int64_t* lld) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    dgt_status st = check_cyclic(h, M, N, mb, nb, p, q, global, ldg, locals, lld);
    if (st != DGT_SUCCESS) return st;
    return launch_block_cyclic(h, true, M, N, mb, nb, p, q, (double*)global, ldg, locals, lld);
}

dgt_status dgt_unpack_block_cyclic(dgt_handle_t h, int64_t M, int64_t N, int64_t mb, int64_t nb, int32_t p,
                                   int32_t q, double* global, int64_t ldg, const double* const* locals,
                                   const int64_t* lld) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    dgt_status st = check_cyclic(h, M, N, mb, nb, p, q, global, ldg, locals, lld);
    if (st != DGT_SUCCESS) return st;
    return launch_block_cyclic(h, false, M, N, mb, nb, p, q, global, ldg, (double* const*)locals, lld);
}

// Device alias of the page-locked host range [p, p + bytes), or nullptr when either end is
// pageable, device memory or not mapped into the device's address space.  Both ends must
// sit in mappings with the same host-to-device offset (one allocation or registration).
static const void* host_range_alias(const void* p, size_t bytes) {
    const char* first = static_cast<const char*>(p);
    const char* last = first + bytes - 1;
    cudaPointerAttributes a0{}, a1{};
    if (cudaPointerGetAttributes(&a0, first) != cudaSuccess || cudaPointerGetAttributes(&a1, last) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a0.type != cudaMemoryTypeHost || a1.type != cudaMemoryTypeHost || !a0.devicePointer || !a1.devicePointer)
        return nullptr;
    if (static_cast<const char*>(a0.devicePointer) - first != static_cast<const char*>(a1.devicePointer) - last)
        return nullptr;
    return a0.devicePointer;
}

// Block-cyclic scatter / gather with the global matrix in page-locked host memory: the
// block_cyclic kernel reads (or writes) the host matrix through its device mapping, so the
// host-device transfer and the permutation are one pass and no device copy of the global
// matrix is made (the reference's full-offload scatter from a host matrix,
// src/Wrappers/cuBLASMp/cuBLASMpWrapped.cpp:633-636, and decompose2D from host A, B, C,
// src/25DCannon.cpp:413-414).
static dgt_status cyclic_host(dgt_context* h, bool to_local, int64_t M, int64_t N, int64_t mb, int64_t nb, int p,
                              int q, const double* global, int64_t ldg, double* const* locals, const int64_t* lld) {
    dgt_status st = check_cyclic(h, M, N, mb, nb, p, q, global, ldg, locals, lld);
    if (st != DGT_SUCCESS) return st;
    if (M == 0 || N == 0) return DGT_SUCCESS;
    const size_t bytes = ((size_t)(N - 1) * (size_t)ldg + (size_t)M) * sizeof(double);
    const void* alias = host_range_alias(global, bytes);
    if (!alias)
        return fail(h, DGT_ERROR_INVALID_VALUE,
                    "global matrix is not page-locked host memory mapped for the device (cudaHostAlloc / cudaHostRegister)");
    return launch_block_cyclic(h, to_local, M, N, mb, nb, p, q, (double*)alias, ldg, locals, lld);
}

dgt_status dgt_pack_block_cyclic_host(dgt_handle_t h, int64_t M, int64_t N, int64_t mb, int64_t nb, int32_t p,
                                      int32_t q, const double* global, int64_t ldg, double* const* locals,
                                      const int64_t* lld) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    return cyclic_host(h, true, M, N, mb, nb, p, q, global, ldg, locals, lld);
}

dgt_status dgt_unpack_block_cyclic_host(dgt_handle_t h, int64_t M, int64_t N, int64_t mb, int64_t nb, int32_t p,
                                        int32_t q, double* global, int64_t ldg, const double* const* locals,
                                        const int64_t* lld) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    return cyclic_host(h, false, M, N, mb, nb, p, q, global, ldg, (double* const*)locals, lld);
}

// One strided copy in the reference's convention: copyBlock swaps rows and columns
// when not column-major (sharedTransfers.cpp:43-44), as does MPI_Type_vector's use.
static HostCopy mk_copy(int64_t rows, int64_t cols, const double* src, int64_t ldS, double* dst, int64_t ldD,
                        bool col_major) {
    if (!col_major) std::swap(rows, cols);
    return HostCopy{src, dst, ldS, ldD, rows, cols};
}

dgt_status dgt_pack_block2d(dgt_handle_t h, int64_t M, int64_t N, int64_t K, int32_t P, int32_t col_major,
                            const double* A, const double* B, const double* C, double* const* lA, double* const* lB,
                            double* const* lC) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (M < 0 || N < 0 || K < 0 || P <= 0) return fail(h, DGT_ERROR_INVALID_VALUE, "bad sizes");
    if (!A || !B || !C || !lA || !lB || !lC) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    int dRow, dCol;
    dgt_block2d_grid(P, &dRow, &dCol);
    if (M < dRow || N < dCol) return fail(h, DGT_ERROR_INVALID_VALUE, "matrix smaller than the grid");
    bool cm = col_major != 0;
    std::vector<HostCopy> copies;
    // deliverMatrix, 2DBlockSequentialDecomposition.cpp:78-144
    for (int i = 0; i < dRow; ++i) {
        int64_t tileM = M / dRow + ((i + 1 == dRow) ? M % dRow : 0);
        for (int j = 0; j < dCol; ++j) {
            int r = i * dCol + j;
            int64_t tileN = N / dCol + ((j + 1 == dCol) ? N % dCol : 0);
            int64_t aOff = (M / dRow) * K * i, bOff = (N / dCol) * j, cOff = (M / dRow) * N * i + (N / dCol) * j;
            int64_t lda = K, ldb = N, ldc = N, llda = K, lldb = tileN, lldc = tileN;
            if (cm) {
                aOff = (M / dRow) * i;
                bOff = (N / dCol) * K * j;
                cOff = (N / dCol) * M * j + (M / dRow) * i;
                lda = M;
                ldb = K;
                ldc = M;
                llda = tileM;
                lldb = K;
                lldc = tileM;
            }
            copies.push_back(mk_copy(tileM, K, A + aOff, lda, lA[r], llda, cm));
            copies.push_back(mk_copy(K, tileN, B + bOff, ldb, lB[r], lldb, cm));
            copies.push_back(mk_copy(tileM, tileN, C + cOff, ldc, lC[r], lldc, cm));
        }
    }
    return launch_strided_copies(h, copies);
}

dgt_status dgt_unpack_block2d(dgt_handle_t h, int64_t M, int64_t N, int32_t P, int32_t col_major, double* C,
                              const double* const* lC) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (M < 0 || N < 0 || P <= 0) return fail(h, DGT_ERROR_INVALID_VALUE, "bad sizes");
    if (!C || !lC) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    int dRow, dCol;
    dgt_block2d_grid(P, &dRow, &dCol);
    if (M < dRow || N < dCol) return fail(h, DGT_ERROR_INVALID_VALUE, "matrix smaller than the grid");
    bool cm = col_major != 0;
    std::vector<HostCopy> copies;
    // gatherResult, 2DBlockSequentialDecomposition.cpp:185-236 (every tile strided; the
    // reference's copyBlock shortcut for rank 0 is not reproduced, see dgt.h)
    for (int i = 0; i < dRow; ++i) {
        int64_t tileM = M / dRow + ((i + 1 == dRow) ? M % dRow : 0);
        for (int j = 0; j < dCol; ++j) {
            int r = i * dCol + j;
            int64_t tileN = N / dCol + ((j + 1 == dCol) ? N % dCol : 0);
            int64_t cOff = (M / dRow) * N * i + (N / dCol) * j, ldc = N, lldc = tileN;
            if (cm) {
                cOff = (N / dCol) * M * j + (M / dRow) * i;
                ldc = M;
                lldc = tileM;
            }
            copies.push_back(mk_copy(tileM, tileN, lC[r], lldc, C + cOff, ldc, cm));
        }
    }
    return launch_strided_copies(h, copies);
}

dgt_status dgt_pack_cannon2d(dgt_handle_t h, int64_t M, int32_t p, const double* A, const double* B,
                             const double* C, double* const* lA, double* const* lB, double* const* lC) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (p <= 0 || M <= 0 || M % p != 0) return fail(h, DGT_ERROR_INVALID_VALUE, "need M % p == 0");
    if (!A || !B || !C || !lA || !lB || !lC) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    const int64_t lm = M / p;
    std::vector<HostCopy> copies;
    // decompose2D, src/25DCannon.cpp:113-136: tile (i,j) at &X[lm*(j*M + i)], ld M
    for (int i = 0; i < p; ++i)
        for (int j = 0; j < p; ++j) {
            int r = i * p + j;
            int64_t off = lm * (j * M + i);
            copies.push_back(HostCopy{A + off, lA[r], M, lm, lm, lm});
            copies.push_back(HostCopy{B + off, lB[r], M, lm, lm, lm});
            copies.push_back(HostCopy{C + off, lC[r], M, lm, lm, lm});
        }
    return launch_strided_copies(h, copies);
}

dgt_status dgt_unpack_cannon2d(dgt_handle_t h, int64_t M, int32_t p, double* C, const double* const* lC) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (p <= 0 || M <= 0 || M % p != 0) return fail(h, DGT_ERROR_INVALID_VALUE, "need M % p == 0");
    if (!C || !lC) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    const int64_t lm = M / p;
    std::vector<HostCopy> copies;
    // reorderMatrix, src/25DCannon.cpp:254-271
    for (int i = 0; i < p; ++i)
        for (int j = 0; j < p; ++j) copies.push_back(HostCopy{lC[i * p + j], C + lm * (j * M + i), lm, M, lm, lm});
    return launch_strided_copies(h, copies);
}

// The Cannon and 2D-block layouts with the global matrices in page-locked host memory: the
// same strided-copy kernels read (or write) the host matrices through their device mapping,
// so the host-device transfer and the permutation are one pass (decompose2D from host A, B,
// C in the full-offload driver, src/25DCannon.cpp:413-414; deliverMatrix / gatherResult
// from a host matrix).  A matrix of 0 bytes is passed through untouched (nothing is read).
static bool alias_all(std::initializer_list<std::pair<const double**, size_t>> xs) {
    for (auto& x : xs) {
        if (x.second == 0) continue;
        const void* a = host_range_alias(*x.first, x.second);
        if (!a) return false;
        *x.first = static_cast<const double*>(a);
    }
    return true;
}
static const char* kNotPinned =
    "global matrix is not page-locked host memory mapped for the device (cudaHostAlloc / cudaHostRegister)";

dgt_status dgt_pack_cannon2d_host(dgt_handle_t h, int64_t M, int32_t p, const double* A, const double* B,
                                  const double* C, double* const* lA, double* const* lB, double* const* lC) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (p <= 0 || M <= 0 || M % p != 0) return fail(h, DGT_ERROR_INVALID_VALUE, "need M % p == 0");
    if (!A || !B || !C || !lA || !lB || !lC) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    const size_t bytes = (size_t)M * (size_t)M * sizeof(double);
    if (!alias_all({{&A, bytes}, {&B, bytes}, {&C, bytes}})) return fail(h, DGT_ERROR_INVALID_VALUE, kNotPinned);
    return dgt_pack_cannon2d(h, M, p, A, B, C, lA, lB, lC);
}

dgt_status dgt_unpack_cannon2d_host(dgt_handle_t h, int64_t M, int32_t p, double* C, const double* const* lC) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (p <= 0 || M <= 0 || M % p != 0) return fail(h, DGT_ERROR_INVALID_VALUE, "need M % p == 0");
    if (!C || !lC) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    const double* c = C;
    if (!alias_all({{&c, (size_t)M * (size_t)M * sizeof(double)}})) return fail(h, DGT_ERROR_INVALID_VALUE, kNotPinned);
    return dgt_unpack_cannon2d(h, M, p, const_cast<double*>(c), lC);
}

dgt_status dgt_pack_block2d_host(dgt_handle_t h, int64_t M, int64_t N, int64_t K, int32_t P, int32_t col_major,
                                 const double* A, const double* B, const double* C, double* const* lA,
                                 double* const* lB, double* const* lC) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (M < 0 || N < 0 || K < 0 || P <= 0) return fail(h, DGT_ERROR_INVALID_VALUE, "bad sizes");
    if (!A || !B || !C || !lA || !lB || !lC) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    const size_t e = sizeof(double);
    if (!alias_all({{&A, (size_t)M * K * e}, {&B, (size_t)K * N * e}, {&C, (size_t)M * N * e}}))
        return fail(h, DGT_ERROR_INVALID_VALUE, kNotPinned);
    return dgt_pack_block2d(h, M, N, K, P, col_major, A, B, C, lA, lB, lC);
}

dgt_status dgt_unpack_block2d_host(dgt_handle_t h, int64_t M, int64_t N, int32_t P, int32_t col_major, double* C,
                                   const double* const* lC) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (M < 0 || N < 0 || P <= 0) return fail(h, DGT_ERROR_INVALID_VALUE, "bad sizes");
    if (!C || !lC) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    const double* c = C;
    if (!alias_all({{&c, (size_t)M * N * sizeof(double)}})) return fail(h, DGT_ERROR_INVALID_VALUE, kNotPinned);
    return dgt_unpack_block2d(h, M, N, P, col_major, const_cast<double*>(c), lC);
}

dgt_status dgt_copy_block(dgt_handle_t h, int64_t rows, int64_t cols, const double* src, double* dst, int64_t ldS,
                          int64_t ldD, int32_t col_major) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (rows < 0 || cols < 0) return fail(h, DGT_ERROR_INVALID_VALUE, "negative size");
    if (rows * cols == 0) return DGT_SUCCESS;  // copyBlock returns early (sharedTransfers.cpp:38-39)
    if (!src || !dst) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    HostCopy c = mk_copy(rows, cols, src, ldS, dst, ldD, col_major != 0);
    if (ldS < c.rows || ldD < c.rows) return fail(h, DGT_ERROR_INVALID_VALUE, "leading dimension < run length");
    return launch_strided_copies(h, {c});
}

dgt_status dgt_copy_block_f32(dgt_handle_t h, int64_t rows, int64_t cols, const float* src, float* dst, int64_t ldS,
                              int64_t ldD, int32_t col_major) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (rows < 0 || cols < 0) return fail(h, DGT_ERROR_INVALID_VALUE, "negative size");
    if (rows * cols == 0) return DGT_SUCCESS;
    if (!src || !dst) return fail(h, DGT_ERROR_INVALID_VALUE, "null pointer");
    if (((uintptr_t)src | (uintptr_t)dst) & 3) return fail(h, DGT_ERROR_INVALID_VALUE, "float pointer not 4-byte aligned");
    if (!col_major) std::swap(rows, cols);
    if (ldS < rows || ldD < rows) return fail(h, DGT_ERROR_INVALID_VALUE, "leading dimension < run length");
    return launch_strided_copy_f32(h, src, dst, ldS, ldD, rows, cols);
}

}  // extern "C"
