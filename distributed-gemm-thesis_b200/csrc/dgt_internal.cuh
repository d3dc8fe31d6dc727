// Shared internals of libdgt: the handle, status plumbing, workspace and the device
// error word that bounded waits report into.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <tuple>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dgt.h"

// Device error word bits (set by kernels, read by dgt_check_device).
#define DGT_DEVERR_TIMEOUT 0x1u
#define DGT_DEVERR_BOUNDS 0x2u

namespace dgt {
// Autotuner table: shape class -> chosen kernel (autotune.cu).
struct TuneKey {
    int mode, lm, ln, lk;  // mode and ceil(log2) of m, n, k
    bool operator<(const TuneKey& o) const {
        return std::tie(mode, lm, ln, lk) < std::tie(o.mode, o.lm, o.ln, o.lk);
    }
};
struct TuneEntry {
    int mode, variant, slices;
    float ms;
    double rel_diff;
};
}  // namespace dgt

struct dgt_context {
    cudaStream_t stream = nullptr;
    int device = 0;
    int num_sms = 148;
    dgt_fp64_mode fp64_mode = DGT_FP64_NATIVE;
    int slices = 7;
    int dmma_variant = 18; // native FP64 kernel variant (see dgemm_dmma.cu): 18 measured fastest for
                           // one plain GEMM; calls outside its TMA form run variant 23 (grouped, decoupled)
    int ozaki_variant = 6; // INT8 Ozaki kernel variant (dgt.h); 6 measured fastest at 16384^3
    bool profile = false;  // record phase events (DGT_TUNE_PROFILE)
    int test_stall = 0;    // failure-path test hook (DGT_TUNE_TEST_STALL)
    bool fuse_steps = true; // DGT_TUNE_FUSE_STEPS
    int crt_panels = 0;     // DGT_TUNE_CRT_PANELS (0: the library's choice)
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};  // split start, gemm start, gemm end
    bool ev_split = false;  // last call had a split phase
    std::string last_error;
    unsigned int* dev_error = nullptr;  // one word in device memory
    // workspace slots: 0 = split planes of the Ozaki / FP32 split paths, 1 = autotuner and
    // probes, 2 = the 2.5D stacks' partial C tiles (live across the Ozaki calls of a Cannon
    // step), 3 = device copies of host operands (dgt_dgemm_host)
    void* ws[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t ws_bytes[4] = {0, 0, 0, 0};
    // dgt_dgemm_host: copy-in and copy-out streams and its events, created on first use
    cudaStream_t copy_stream[2] = {nullptr, nullptr};
    cudaEvent_t copy_ev[24] = {};
    // the CRT product in op(B) panels: split and reconstruction streams and their events,
    // created on first use
    cudaStream_t work_stream[2] = {nullptr, nullptr};
    cudaEvent_t work_ev[1 + 3 * 8] = {};
    std::atomic<int64_t> launches{0};
    std::map<dgt::TuneKey, dgt::TuneEntry> tune;
    // device copies of launch tables (grouped problems, Ozaki jobs and schedules), keyed by
    // a hash of their content (see device_table)
    struct DevTable {
        uint64_t hash;
        size_t bytes;
        void* ptr;
        uint64_t last_use;
    };
    std::vector<DevTable> tables;
    uint64_t table_clock = 0;
};

namespace dgt {

// Opts Kernel into `bytes` of dynamic shared memory on the current device.  The attribute
// belongs to the device's context, so it is set once per (kernel, device) -- a process that
// launches on several devices sets it on each -- under a mutex, since host threads may
// launch concurrently.
template <auto Kernel>
cudaError_t smem_opt_in(int bytes) {
    constexpr int kMaxDev = 64;
    static std::mutex mu;
    static bool done[kMaxDev] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev)
        return cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    std::lock_guard<std::mutex> g(mu);
    if (!done[dev]) {
        e = cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
        done[dev] = true;
    }
    return cudaSuccess;
}

inline dgt_status fail(dgt_context* h, dgt_status s, const std::string& msg) {
    if (h) h->last_error = msg;
    return s;
}

inline dgt_status cuda_fail(dgt_context* h, cudaError_t e, const char* what) {
    return fail(h, DGT_ERROR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define DGT_CUDA_TRY(h, call)                                     \
    do {                                                          \
        cudaError_t _e = (call);                                  \
        if (_e != cudaSuccess) return dgt::cuda_fail(h, _e, #call); \
    } while (0)

#define DGT_LAUNCH_CHECK(h, name)                                          \
    do {                                                                   \
        (h)->launches.fetch_add(1);                                        \
        cudaError_t _e = cudaGetLastError();                               \
        if (_e != cudaSuccess) return dgt::cuda_fail(h, _e, name " launch"); \
    } while (0)

// Phase markers for DGT_TUNE_PROFILE (no-ops unless profiling is on).
void mark(dgt_context* h, int which);

// Device copy of a host table made of n parts, part i placed at offsets[i] (256-byte
// aligned), taken from a per-handle cache keyed by a hash of the content: a repeated call
// (one replayed from a captured CUDA graph among them) finds its table resident and issues
// no copy.  Up to kMaxDeviceTables tables stay resident; beyond that the least recently used
// one is released (after the handle's stream drains).
constexpr int kMaxDeviceTables = 64;
dgt_status device_table(dgt_context* h, int n, const void* const* parts, const size_t* bytes, void** out,
                        size_t* offsets);

// Grows a handle-owned scratch buffer; never shrinks.  slot 0, 1 or 2.
dgt_status ensure_workspace(dgt_context* h, size_t bytes, void** out, int slot = 0);

inline bool is_trans(char t) { return t == 'T' || t == 't' || t == 'C' || t == 'c'; }
// slices: digit slices of the Ozaki slice scheme, or moduli of the CRT scheme
inline bool valid_slices(dgt_fp64_mode mode, int slices) {
    return mode == DGT_FP64_OZAKI2_INT8 ? (slices >= 8 && slices <= 20) : (slices >= 2 && slices <= 16);
}
inline bool valid_op(char t) { return t == 'N' || t == 'n' || is_trans(t); }

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// ---- native FP64 GEMM engine (dgemm_dmma.cu) --------------------------------------------
// One K-segment: C += op(A_seg) * op(B_seg) over k rows/cols.  A problem is a list of
// segments that accumulate into the same C tile (the SUMMA / Cannon step schedule).
struct KSegment {
    const double* A;
    const double* B;
    int64_t lda, ldb;
    int64_t k;
};

struct Problem {
    int64_t m, n;
    double alpha, beta;
    double* C;
    int64_t ldc;
    int32_t seg_begin, seg_count;  // into the segment table
    int32_t transa, transb;        // 0 = 'N', 1 = 'T'
    int32_t tile_begin;            // prefix sum of tiles (filled by the launcher)
    int32_t tiles_m, tiles_n;
    // Stack reduction inside the launch (2.5D Cannon).  red_role 1: a partial problem; it stores
    // its tiles, then counts each in red_flags[red_slot + local tile].  red_role 2: a stack-0
    // problem; it waits until its tile's count reaches red_wait and adds the red_wait partial
    // tiles red_src + s * red_stride (leading dimension red_ld), s = 0, 1, ..., to its own
    // result in that order.  Partial problems' tiles are numbered before every stack-0 tile,
    // which, with all CTAs resident, keeps every wait finite.  red_role 0: no reduction.
    const double* red_src;
    int64_t red_stride, red_ld;
    int32_t red_role, red_slot, red_wait, red_pad;
};

int dmma_variant_count();
int64_t dmma_tile_count(int64_t m, int64_t n);  // CTA tiles of one m x n problem of the grouped kernel
TuneKey tune_key(int mode, int64_t m, int64_t n, int64_t k);
const TuneEntry* tune_lookup(dgt_context* h, int mode, int64_t m, int64_t n, int64_t k);
// Argument checks shared by the GEMM entry points (api.cu).
dgt_status validate_gemm(dgt_context* h, char ta, char tb, int64_t m, int64_t n, int64_t k, const void* A,
                         int64_t lda, const void* B, int64_t ldb, const void* C, int64_t ldc);
// Launches the persistent grouped FP64 DMMA kernel over problems/segments (host arrays,
// copied to device workspace).  Validation is the caller's job.
// red_flags: the stack-reduction counters (zeroed by the launcher), or null when no problem
// reduces.
dgt_status launch_dmma_grouped(dgt_context* h, std::vector<Problem>& probs, const std::vector<KSegment>& segs,
                               int32_t* red_flags = nullptr, size_t red_count = 0);

// ---- layout engine (layout.cu) ---------------------------------------------------------
// One strided copy: rows x cols, column-major (rows contiguous on both sides).
struct HostCopy {
    const double* src;
    double* dst;
    int64_t ldS, ldD, rows, cols;
};
dgt_status launch_block_cyclic(dgt_context* h, bool to_local, int64_t M, int64_t N, int64_t mb, int64_t nb, int p,
                               int q, double* global, int64_t ldg, double* const* locals, const int64_t* lld);
dgt_status launch_strided_copies(dgt_context* h, const std::vector<HostCopy>& copies);
dgt_status launch_strided_copy_f32(dgt_context* h, const float* src, float* dst, int64_t ldS, int64_t ldD,
                                   int64_t rows, int64_t cols);
// C[e] += parts[0][e] + ... + parts[nparts-1][e] (plain loads: parts may be peer memory).
dgt_status launch_tile_sum(dgt_context* h, double* C, const double* const* parts, int nparts, int64_t elems);
// C[t] += sum_{s < stacks} W[s*stack_stride + t*elems_per_tile + e] for every tile t.
dgt_status launch_stack_reduce(dgt_context* h, int64_t elems_per_tile, int tiles, int stacks, double* const* C,
                               const double* W, int64_t stack_stride);

// ---- Ozaki emulation (ozaki.cu) -----------------------------------------------------------
// Scratch bytes one INT8 Ozaki call needs (0 if the shape is unsupported).
size_t ozaki_scratch_bytes(int S, int64_t m, int64_t n, int64_t k);
// Workspace upper bounds over kernel variants (dgt_dgemm_workspace_size).
dgt_status ozaki_workspace_bound(int S, int64_t m, int64_t n, int64_t k, bool bf16, size_t* bytes);
dgt_status ozaki2_workspace_bound(int nmod, int64_t m, int64_t n, int64_t k, size_t* bytes);
// The INT8 Ozaki path on caller-provided scratch; no allocation, no handle.
dgt_status ozaki_dgemm_on(cudaStream_t s, int num_sms, unsigned int* err, void* ws, size_t ws_bytes, bool ta,
                          bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                          const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int S);
dgt_status ozaki_dgemm(dgt_context* h, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                       const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc,
                       dgt_fp64_mode mode, int slices);

// Per-row (or per-column) max |x| of op(A) / op(B)^T as the bit pattern of |x|, one word per
// row; kcontig: element (mn, kk) at X[kk + mn*ld], else at X[mn + kk*ld].
dgt_status ozaki_amax(dgt_context* h, cudaStream_t s, const double* X, int64_t ld, int64_t MN, int64_t K,
                      bool kcontig, unsigned long long* out);
// FP64-accurate GEMM by CRT over INT8 residues (ozaki2.cu); nmod = number of moduli.
dgt_status ozaki2_dgemm(dgt_context* h, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                        const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                        int64_t ldc, int nmod);

// One product of a grouped Ozaki launch (all sizes > 0; validation is the caller's job).
struct OzProblem {
    bool ta, tb;
    int64_t m, n, k;
    double alpha, beta;
    const double* A;
    int64_t lda;
    const double* B;
    int64_t ldb;
    double* C;
    int64_t ldc;
    // CRT scheme only.  nseg > 0: K is the concatenation of the pieces segs[0 .. nseg) (each
    // with its own A, B, lda, ldb and k > 0; k above is their total, A and B are unused): one
    // product, its rows and columns scaled over the whole K, so a step schedule's steps
    // become one exact residue sum.  stack 1: a further stack of the preceding product's
    // output (same m, n, C and ldc, beta 0); alpha times its result is added to the preceding
    // stacks' sum, in order (the 2.5D stack reduction).
    const KSegment* segs = nullptr;
    int32_t nseg = 0;
    int32_t stack = 0;
};
// All products in one INT8 emulation pass: one amax launch, one split launch, one persistent
// GEMM launch over every product's tiles (and, for the CRT scheme, one reconstruction
// launch).  slices = digit slices, or moduli when crt.  Returns DGT_ERROR_UNSUPPORTED (with
// no work issued) when a product's K is too long for the grouped form; the caller then runs
// the products one by one.
dgt_status ozaki_dgemm_grouped(dgt_context* h, const std::vector<OzProblem>& probs, int slices, bool crt);

}  // namespace dgt
