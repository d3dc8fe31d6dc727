// FP64-accurate GEMM emulated on the INT8 tensor cores of sm_100a (Ozaki scheme I,
// integer slices: Ozaki, Ogita, Oishi, Rump 2012; INT8 form: Ootomo, Ozaki, Yokota 2024).
//
//   1. Scale: every row i of op(A) gets e_i with max_k |a_ik| in [2^(e_i-1), 2^e_i), every
//      column j of op(B) gets f_j likewise, so a_ik * 2^-e_i lies in (-1, 1).
//   2. Split: v = a * 2^(7-e) is cut into S truncated 7-bit digits s_1..s_S in [-127, 127]
//      (v = s_1 + r_1, r_1 * 2^7 = s_2 + r_2, ...): a = 2^e * sum_s s_s 2^(-7s) + O(2^(e-7S)).
//      Every step is exact in FP64.  Digits are stored as K-major INT8 planes.
//   3. Multiply: for each diagonal d = s + t (2 <= d <= S+1) the digit products
//      P_d = sum_{s+t=d} A_s B_t are accumulated EXACTLY in INT32 in tensor memory by
//      tcgen05.mma kind::i8 (|P_d| <= pairs * 127^2 * K < 2^31 is enforced by chunking
//      the diagonal into flush groups).
//   4. Recombine in FP64: C = beta*C + alpha * sum_d 2^(e_i + f_j - 7d) P_d, least
//      significant diagonal first; one FP64 rounding per flush group.
//
// The FLOP count reported for this path is 2*M*N*K FP64-equivalent flops, whatever S is.
//
// GEMM kernel: persistent, one 128 x 256 output tile per CTA at a time, warp-specialised:
// warp 0 issues TMA loads of the digit planes (128B-swizzled, 4-stage ring), warp 1 issues
// tcgen05.mma into one of two 256-column INT32 accumulators in TMEM, warps 2-5 drain the
// other accumulator (tcgen05.ld) into C in FP64 while the next group multiplies.  Every
// mbarrier wait has an iteration budget; on expiry the kernel records DGT_DEVERR_TIMEOUT,
// stops all roles, waits for its own MMAs, frees TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <vector>

#include "crt.cuh"
#include "dgt_internal.cuh"
#include "tc_engine.cuh"

namespace dgt {
namespace oz {

// MN-contiguous operand: element (mn, kk) at X[mn + kk*ld]; one thread per mn, K split over
// blocks (bx covers 256 mn, by a chunk of K).
__device__ __forceinline__ void amax_mn_block(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                              int kchunk, unsigned long long* __restrict__ amax, int64_t bx,
                                              int64_t by) {
    int64_t mn = bx * blockDim.x + threadIdx.x;
    if (mn >= MN) return;
    int64_t k0 = by * kchunk, k1 = min(K, k0 + kchunk);
    unsigned long long mx = 0;
    for (int64_t kk = k0; kk < k1; ++kk) {
        unsigned long long b = (unsigned long long)__double_as_longlong(X[mn + kk * ld]) & 0x7fffffffffffffffull;
        mx = b > mx ? b : mx;
    }
    if (mx) atomicMax(amax + mn, mx);
}

__global__ void amax_mn_contig(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K, int kchunk,
                               unsigned long long* __restrict__ amax) {
    amax_mn_block(X, ld, MN, K, kchunk, amax, blockIdx.x, blockIdx.y);
}

// K-contiguous operand: element (mn, kk) at X[kk + mn*ld]; one warp per mn.  atomic: the row
// may have other pieces (amax zeroed by the caller), so the result goes in by atomicMax.
__device__ __forceinline__ void amax_k_block(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                             unsigned long long* __restrict__ amax, int64_t bx,
                                             bool atomic = false) {
    int64_t mn = bx * (blockDim.x / 32) + threadIdx.x / 32;
    int lane = threadIdx.x & 31;
    if (mn >= MN) return;
    const double* row = X + mn * ld;
    unsigned long long mx = 0;
    for (int64_t kk = lane; kk < K; kk += 32) {
        unsigned long long b = (unsigned long long)__double_as_longlong(row[kk]) & 0x7fffffffffffffffull;
        mx = b > mx ? b : mx;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        unsigned long long other = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = other > mx ? other : mx;
    }
    if (lane == 0) {
        if (!atomic)
            amax[mn] = mx;
        else if (mx)
            atomicMax(amax + mn, mx);
    }
}

__global__ void amax_k_contig(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                              unsigned long long* __restrict__ amax) {
    amax_k_block(X, ld, MN, K, amax, blockIdx.x);
}

// Digit planes: plane s holds digit s+1 of every element as int8 at [s][mn][kk] (K-major,
// row length k_pad, mn_pad rows); padding rows/columns are written as 0.  Each thread
// produces 32 consecutive kk of one mn (block bx covers 128 mn, by 32 of K).  The by == 0
// blocks also write exps[mn].  BF16OUT stores each digit as a BF16 value instead (exact:
// |digit| <= 127 < 2^8), two bytes per element.
template <bool K_CONTIG, bool BF16OUT>
__device__ __forceinline__ void split_block(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                            int64_t mn_pad, int64_t k_pad, int S,
                                            const unsigned long long* __restrict__ amax, int32_t* __restrict__ exps,
                                            void* __restrict__ planes_v, int64_t bx, int64_t by) {
    const int64_t mn = bx * blockDim.x + threadIdx.x;
    const int64_t k0 = by * 32;
    if (mn >= mn_pad) return;
    double v[32];
    int e = 0;
    if (mn < MN) {
        e = exponent_of_max(amax[mn]);
        if (by == 0) exps[mn] = e;
    }
    const bool live = (mn < MN) && (e != EXP_NONFINITE);
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        int64_t kk = k0 + i;
        double x = 0.0;
        if (live && kk < K) x = K_CONTIG ? X[kk + mn * ld] : X[mn + kk * ld];
        v[i] = live ? scale2(x, 7 - e) : 0.0;  // in (-128, 128)
    }
    const int64_t plane = mn_pad * k_pad;
    for (int s = 0; s < S; ++s) {
        if constexpr (!BF16OUT) {
            uint32_t w[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) w[q] = 0;
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                int dgt = __double2int_rz(v[i]);       // truncation toward zero: |dgt| <= 127
                v[i] = (v[i] - (double)dgt) * 128.0;  // exact remainder, rescaled
                w[i >> 2] |= ((uint32_t)(uint8_t)(int8_t)dgt) << (8 * (i & 3));
            }
            uint4* o4 = reinterpret_cast<uint4*>((int8_t*)planes_v + s * plane + mn * k_pad + k0);
            o4[0] = make_uint4(w[0], w[1], w[2], w[3]);
            o4[1] = make_uint4(w[4], w[5], w[6], w[7]);
        } else {
            uint32_t w[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) w[q] = 0;
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                int dgt = __double2int_rz(v[i]);
                v[i] = (v[i] - (double)dgt) * 128.0;
                // an integer of at most 7 bits: its BF16 pattern is exact
                const uint32_t b = (uint32_t)__bfloat16_as_ushort(__int2bfloat16_rn(dgt));
                w[i >> 1] |= b << (16 * (i & 1));
            }
            uint4* o4 = reinterpret_cast<uint4*>((__nv_bfloat16*)planes_v + s * plane + mn * k_pad + k0);
#pragma unroll
            for (int q = 0; q < 4; ++q) o4[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
        }
    }
}

template <bool K_CONTIG, bool BF16OUT>
__global__ void __launch_bounds__(128) split_digits(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                                    int64_t mn_pad, int64_t k_pad, int S,
                                                    const unsigned long long* __restrict__ amax,
                                                    int32_t* __restrict__ exps, void* __restrict__ planes_v) {
    split_block<K_CONTIG, BF16OUT>(X, ld, MN, K, mn_pad, k_pad, S, amax, exps, planes_v, blockIdx.x, blockIdx.y);
}

// ---- grouped pre-pass: one launch scales (or splits) every operand of a grouped call -------
__global__ void __launch_bounds__(256) amax_grouped(const SplitJob* __restrict__ jobs, int njobs) {
    const int64_t blk = blockIdx.x;
    const SplitJob& J = jobs[find_job(jobs, njobs, blk, false)];
    const int64_t local = blk - J.amax_begin;
    if (J.kcontig)
        amax_k_block(J.X, J.ld, J.MN, J.K, J.amax, local, true);
    else
        amax_mn_block(J.X, J.ld, J.MN, J.K, AMAX_KCHUNK, J.amax, local % J.amax_bx, local / J.amax_bx);
}

__global__ void __launch_bounds__(128) split_grouped(const SplitJob* __restrict__ jobs, int njobs, int S) {
    const int64_t blk = blockIdx.x;
    const SplitJob& J = jobs[find_job(jobs, njobs, blk, true)];
    const int64_t local = blk - J.split_begin;
    const int64_t bx = local % J.split_bx, by = local / J.split_bx;
    if (J.kcontig)
        split_block<true, false>(J.X, J.ld, J.MN, J.K, J.mn_pad, J.k_pad, S, J.amax, J.exps, J.planes, bx, by);
    else
        split_block<false, false>(J.X, J.ld, J.MN, J.K, J.mn_pad, J.k_pad, S, J.amax, J.exps, J.planes, bx, by);
}

// ---- the INT8 tcgen05 GEMM ---------------------------------------------------------------------


}  // namespace oz

// Builds the flush-group schedule: diagonals from least to most significant.
//  INT8 digits: a group holds as many pairs of a diagonal as keep
//               pairs * 127^2 * k_pad < 2^31 (exact INT32 accumulation), over all of K.
//  BF16 digits: FP32 accumulation is exact only below 2^24, so every pair is flushed after
//               at most 1024 elements of K (127^2 * 1024 < 2^24): one group per pair and chunk.
// Segment k-ranges are in units of one pipeline stage (tkb bytes).
static bool ozaki_schedule(int S, int64_t k_pad, int tkb, bool bf16, std::vector<oz::Seg>& segs,
                           std::vector<oz::Group>& groups) {
    const int esize = bf16 ? 2 : 1;
    const int64_t kb = k_pad * esize / tkb;
    for (int d = S + 1; d >= 2; --d) {  // 1-based digit indices s + t = d
        std::vector<std::pair<int, int>> pairs;
        for (int s = 1; s <= S; ++s) {
            int t = d - s;
            if (t >= 1 && t <= S) pairs.emplace_back(s - 1, t - 1);
        }
        if (!bf16) {
            const int64_t per_pair = 127LL * 127LL * k_pad;
            if (per_pair > (int64_t)INT32_MAX) return false;
            const int max_pairs = (int)std::max<int64_t>(1, (int64_t)INT32_MAX / per_pair);
            for (size_t i = 0; i < pairs.size(); i += max_pairs) {
                oz::Group g{(int32_t)segs.size(), 0, d, 0};
                for (size_t j = i; j < std::min(pairs.size(), i + (size_t)max_pairs); ++j)
                    segs.push_back(oz::Seg{pairs[j].first, pairs[j].second, 0, (int32_t)kb});
                g.seg1 = (int32_t)segs.size();
                groups.push_back(g);
            }
        } else {
            const int64_t chunk_kb = 1024 * esize / tkb;  // 1024 elements of K per flush
            for (auto& pr : pairs)
                for (int64_t c = 0; c < kb; c += chunk_kb) {
                    oz::Group g{(int32_t)segs.size(), 0, d, 0};
                    segs.push_back(oz::Seg{pr.first, pr.second, (int32_t)c, (int32_t)std::min(kb, c + chunk_kb)});
                    g.seg1 = (int32_t)segs.size();
                    groups.push_back(g);
                }
        }
    }
    return true;
}

// Scratch layout of one Ozaki call: planes A | planes B | amax A | amax B | exp A | exp B |
// schedule.  Returns false when the shape is outside what the kernels support.
struct OzakiLayout {
    int64_t m_pad, n_pad, k_pad;
    int variant, tkb;
    bool bf16;
    size_t pa, pb, xa, xb, ea, eb, sb, gb, total;
    std::vector<oz::Seg> segs;
    std::vector<oz::Group> groups;
};

// variant: 0 = 4 epilogue warps / 128-byte stages x4, 1 = 8 warps / 128 B x4,
//          2 = 4 warps / 64 B x8, 3 = 8 warps / 64 B x8,
//          4 = CTA pair (cta_group::2, 256 x 256 tiles), 8 warps / 128 B x6
static int variant_tkb(int variant) { return (variant == 2 || variant == 3) ? 64 : 128; }
static bool variant_pair(int variant) { return variant == 4; }

static dgt_status ozaki_layout(dgt_context* h, int S, int64_t m, int64_t n, int64_t k, int variant, bool bf16,
                               OzakiLayout& L) {
    L.variant = variant;
    L.bf16 = bf16;
    L.tkb = variant_tkb(variant);
    const int64_t m_unit = variant_pair(variant) ? 2 * oz::TM : oz::TM;
    L.m_pad = ceil_div(m, m_unit) * m_unit;
    L.n_pad = ceil_div(n, oz::TN) * oz::TN;
    L.k_pad = ceil_div(k, oz::KPAD) * oz::KPAD;
    if (!ozaki_schedule(S, L.k_pad, L.tkb, bf16, L.segs, L.groups))
        return fail(h, DGT_ERROR_UNSUPPORTED, "K too large for exact INT32 accumulation of one digit product");
    if ((int64_t)S * std::max(L.m_pad, L.n_pad) > INT32_MAX)
        return fail(h, DGT_ERROR_UNSUPPORTED, "matrix too large for 32-bit TMA coordinates");
    auto up = [](size_t x) { return (x + 1023) / 1024 * 1024; };
    const size_t esize = bf16 ? 2 : 1;
    L.pa = up((size_t)S * L.m_pad * L.k_pad * esize);
    L.pb = up((size_t)S * L.n_pad * L.k_pad * esize);
    L.xa = up(m * 8);
    L.xb = up(n * 8);
    L.ea = up(m * 4);
    L.eb = up(n * 4);
    L.sb = up(L.segs.size() * sizeof(oz::Seg));
    L.gb = up(L.groups.size() * sizeof(oz::Group));
    L.total = L.pa + L.pb + L.xa + L.xb + L.ea + L.eb + L.sb + L.gb;
    return DGT_SUCCESS;
}

// Largest workspace of the slice scheme over the kernel variants (0 .. 4) for this shape;
// DGT_ERROR_UNSUPPORTED when no variant can run it.
dgt_status ozaki_workspace_bound(int S, int64_t m, int64_t n, int64_t k, bool bf16, size_t* bytes) {
    size_t best = 0;
    bool any = false;
    for (int v = 0; v <= 4; ++v) {
        OzakiLayout L;
        if (ozaki_layout(nullptr, S, m, n, k, v, bf16, L) != DGT_SUCCESS) continue;
        best = std::max(best, L.total);
        any = true;
    }
    *bytes = best;
    return any ? DGT_SUCCESS : DGT_ERROR_UNSUPPORTED;
}

size_t ozaki_scratch_bytes(int S, int64_t m, int64_t n, int64_t k) {
    OzakiLayout L;
    return ozaki_layout(nullptr, S, m, n, k, 0, false, L) == DGT_SUCCESS ? L.total : 0;
}

template <class CF, int KIND>
static cudaError_t launch_ozaki_variant(const CUtensorMap& tmA, const CUtensorMap& tmB, const oz::Params& prm,
                                        int num_sms, cudaStream_t s) {
    cudaError_t e = smem_opt_in<oz::digit_gemm<CF, KIND, 0>>((int)CF::SMEM);
    if (e != cudaSuccess) return e;
    const int tiles = prm.tiles_m * prm.tiles_n;
    if constexpr (CF::PAIR) {
        // one 2-CTA cluster per 256 x 256 tile, persistent over half the SMs' worth of clusters
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(2 * std::min(tiles, num_sms / 2)));
        cfg.blockDim = dim3(CF::THREADS);
        cfg.dynamicSmemBytes = CF::SMEM;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 2;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, oz::digit_gemm<CF, KIND, 0>, tmA, tmB, prm);
    } else {
        oz::digit_gemm<CF, KIND, 0><<<std::min(tiles, num_sms), CF::THREADS, CF::SMEM, s>>>(tmA, tmB, prm);
        return cudaGetLastError();
    }
}

// The Ozaki INT8 path on caller-provided scratch (L.total bytes at ws).  h may be null:
// then no profiling marks, launch counts or error messages are recorded.
static dgt_status ozaki_run(dgt_context* h, cudaStream_t s, int num_sms, unsigned int* err, void* ws,
                            const OzakiLayout& L, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                            const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                            int64_t ldc, int S) {
    const int64_t m_pad = L.m_pad, n_pad = L.n_pad, k_pad = L.k_pad;
    char* p = (char*)ws;
    void* planesA = p;
    void* planesB = p + L.pa;
    unsigned long long* amaxA = (unsigned long long*)(p + L.pa + L.pb);
    unsigned long long* amaxB = (unsigned long long*)(p + L.pa + L.pb + L.xa);
    int32_t* expA = (int32_t*)(p + L.pa + L.pb + L.xa + L.xb);
    int32_t* expB = (int32_t*)(p + L.pa + L.pb + L.xa + L.xb + L.ea);
    oz::Seg* dsegs = (oz::Seg*)(p + L.pa + L.pb + L.xa + L.xb + L.ea + L.eb);
    oz::Group* dgroups = (oz::Group*)(p + L.pa + L.pb + L.xa + L.xb + L.ea + L.eb + L.sb);
    auto counted = [&](const char* what) -> dgt_status {
        if (h) h->launches.fetch_add(1);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? DGT_SUCCESS : cuda_fail(h, e, what);
    };

    const bool inline_sched = L.segs.size() <= (size_t)oz::MAX_SEGS && L.groups.size() <= (size_t)oz::MAX_GROUPS;
    if (!inline_sched) {  // long BF16 schedules: a device table from the handle's cache
        if (!h) return DGT_ERROR_UNSUPPORTED;
        const void* parts[2] = {L.segs.data(), L.groups.data()};
        const size_t bytes[2] = {L.segs.size() * sizeof(oz::Seg), L.groups.size() * sizeof(oz::Group)};
        size_t offs[2];
        void* table = nullptr;
        dgt_status st = device_table(h, 2, parts, bytes, &table, offs);
        if (st != DGT_SUCCESS) return st;
        dsegs = (oz::Seg*)((char*)table + offs[0]);
        dgroups = (oz::Group*)((char*)table + offs[1]);
    }
    if (h) mark(h, 0);
    // op(A) is m x k: 'N' -> element (i,kk) at A[i + kk*lda] (MN-contiguous); 'T' -> A[kk + i*lda]
    // op(B) as its transpose n x k: 'N' -> element (j,kk) at B[kk + j*ldb] (K-contiguous); 'T' -> B[j + kk*ldb]
    auto amax = [&](const double* X, int64_t ld, int64_t MN, bool kcontig, unsigned long long* out) {
        return ozaki_amax(h, s, X, ld, MN, k, kcontig, out);
    };
    auto split = [&](const double* X, int64_t ld, int64_t MN, int64_t mn_pad, bool kcontig,
                     const unsigned long long* am, int32_t* ex, void* planes) {
        dim3 grid((unsigned)ceil_div(mn_pad, 128), (unsigned)(k_pad / 32));
        if (kcontig && !L.bf16)
            oz::split_digits<true, false><<<grid, 128, 0, s>>>(X, ld, MN, k, mn_pad, k_pad, S, am, ex, planes);
        else if (!L.bf16)
            oz::split_digits<false, false><<<grid, 128, 0, s>>>(X, ld, MN, k, mn_pad, k_pad, S, am, ex, planes);
        else if (kcontig)
            oz::split_digits<true, true><<<grid, 128, 0, s>>>(X, ld, MN, k, mn_pad, k_pad, S, am, ex, planes);
        else
            oz::split_digits<false, true><<<grid, 128, 0, s>>>(X, ld, MN, k, mn_pad, k_pad, S, am, ex, planes);
        return counted("ozaki split");
    };
    dgt_status st;
    if ((st = amax(A, lda, m, ta, amaxA)) != DGT_SUCCESS) return st;
    if ((st = amax(B, ldb, n, !tb, amaxB)) != DGT_SUCCESS) return st;
    if ((st = split(A, lda, m, m_pad, ta, amaxA, expA, planesA)) != DGT_SUCCESS) return st;
    if ((st = split(B, ldb, n, n_pad, !tb, amaxB, expB, planesB)) != DGT_SUCCESS) return st;

    CUtensorMap tmA, tmB;
    const int64_t row_bytes = k_pad * (L.bf16 ? 2 : 1);
    // box heights must equal what one CTA stages per operand: in the CTA-pair kernel each CTA
    // holds only half of B's 256 rows (TN / 2), so its box is 128 rows high
    const int b_box = variant_pair(L.variant) ? oz::TN / 2 : oz::TN;
    if (!oz::make_plane_map(&tmA, planesA, (int64_t)S * m_pad, row_bytes, oz::TM, L.tkb) ||
        !oz::make_plane_map(&tmB, planesB, (int64_t)S * n_pad, row_bytes, b_box, L.tkb))
        return fail(h, DGT_ERROR_CUDA, "cuTensorMapEncodeTiled failed");
    static thread_local oz::Params prm;  // ~21 KB: keep it off the stack
    prm = oz::Params{};
    prm.m = m;
    prm.n = n;
    prm.ldc = ldc;
    prm.m_pad = (int32_t)m_pad;
    prm.n_pad = (int32_t)n_pad;
    prm.tiles_m = (int32_t)(m_pad / (variant_pair(L.variant) ? 2 * oz::TM : oz::TM));
    prm.tiles_n = (int32_t)(n_pad / oz::TN);
    prm.ngroups = (int32_t)L.groups.size();
    prm.alpha = alpha;
    prm.beta = beta;
    prm.C = C;
    prm.row_exp = expA;
    prm.col_exp = expB;
    if (inline_sched) {
        std::copy(L.segs.begin(), L.segs.end(), prm.segs);
        std::copy(L.groups.begin(), L.groups.end(), prm.groups);
        prm.segs_ext = nullptr;
        prm.groups_ext = nullptr;
    } else {
        prm.segs_ext = dsegs;
        prm.groups_ext = dgroups;
    }
    prm.err = err;
    prm.test_stall = (h && h->test_stall == 1) ? 1 : 0;
    const int tiles = prm.tiles_m * prm.tiles_n;
    const int grid = std::min(tiles, num_sms);
    if (h) mark(h, 1);
    cudaError_t le;
    if (L.bf16) {
        le = launch_ozaki_variant<oz::OzCfg<8, 128, 4>, 1>(tmA, tmB, prm, num_sms, s);
    } else {
        switch (L.variant) {
            case 1: le = launch_ozaki_variant<oz::OzCfg<8, 128, 4>, 0>(tmA, tmB, prm, num_sms, s); break;
            case 2: le = launch_ozaki_variant<oz::OzCfg<4, 64, 8>, 0>(tmA, tmB, prm, num_sms, s); break;
            case 3: le = launch_ozaki_variant<oz::OzCfg<8, 64, 8>, 0>(tmA, tmB, prm, num_sms, s); break;
            case 4: le = launch_ozaki_variant<oz::OzCfg<8, 128, 6, true>, 0>(tmA, tmB, prm, num_sms, s); break;
            default: le = launch_ozaki_variant<oz::OzCfg<4, 128, 4>, 0>(tmA, tmB, prm, num_sms, s); break;
        }
    }
    if (h) h->launches.fetch_add(1);
    if (le != cudaSuccess) return cuda_fail(h, le, "ozaki_i8_gemm launch");
    if (h) mark(h, 2);
    return DGT_SUCCESS;
}

dgt_status ozaki_dgemm_on(cudaStream_t s, int num_sms, unsigned int* err, void* ws, size_t ws_bytes, bool ta,
                          bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                          const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int S) {
    OzakiLayout L;
    dgt_status st = ozaki_layout(nullptr, S, m, n, k, 0, false, L);
    if (st != DGT_SUCCESS) return st;
    if (L.total > ws_bytes) return DGT_ERROR_INVALID_VALUE;
    return ozaki_run(nullptr, s, num_sms, err, ws, L, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, S);
}

dgt_status ozaki_dgemm(dgt_context* h, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                       const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                       int64_t ldc, dgt_fp64_mode mode, int S) {
    if (mode != DGT_FP64_OZAKI_INT8 && mode != DGT_FP64_OZAKI_BF16)
        return fail(h, DGT_ERROR_UNSUPPORTED, "unknown Ozaki mode");
    OzakiLayout L;
    // variants 5, 6 and 7 differ from 1, 4 and 0 only in the CRT residue GEMM's unit order; the BF16
    // kernel has a single form (8 epilogue warps, 128-byte stages, one CTA per tile), so its
    // layout is variant 1's whatever the handle's INT8 choice
    const bool bf16 = mode == DGT_FP64_OZAKI_BF16;
    const int hv = h->ozaki_variant;
    const int ov = bf16 ? 1 : hv == 5 ? 1 : hv == 6 ? 4 : hv == 7 ? 0 : hv;
    dgt_status st = ozaki_layout(h, S, m, n, k, ov, bf16, L);
    if (st != DGT_SUCCESS) return st;
    void* ws = nullptr;
    st = ensure_workspace(h, L.total, &ws, 0);
    if (st != DGT_SUCCESS) return st;
    return ozaki_run(h, h->stream, h->num_sms, h->dev_error, ws, L, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C,
                     ldc, S);
}


// ---- grouped: every product of a batch in one pre-pass and one persistent GEMM launch ----------

template <class CF, int EPI>
static cudaError_t launch_ozaki_grouped(const oz::Params& prm, int grid, cudaStream_t s) {
    cudaError_t e = smem_opt_in<oz::digit_gemm<CF, 0, EPI, true>>((int)CF::SMEM);
    if (e != cudaSuccess) return e;
    static const CUtensorMap unused = {};  // grouped mode reads each problem's maps from its table
    oz::digit_gemm<CF, 0, EPI, true><<<grid, CF::THREADS, CF::SMEM, s>>>(unused, unused, prm);
    return cudaGetLastError();
}

dgt_status ozaki_dgemm_grouped(dgt_context* h, const std::vector<OzProblem>& probs, int S, bool crt) {
    const int T = (int)probs.size();
    if (T == 0) return DGT_SUCCESS;
    if (!valid_slices(crt ? DGT_FP64_OZAKI2_INT8 : DGT_FP64_OZAKI_INT8, S))
        return fail(h, DGT_ERROR_INVALID_VALUE, "slice count must be in [2, 16] (moduli: [8, 20])");
    // variants 0 and 1 (4 or 8 epilogue warps, 128-byte stages); 7 runs as 0 and the others as 1,
    // 5, 6 and 7 with the GEMM's units taken in a dynamic order (the heaviest products' tiles are
    // numbered first, and a CTA that finishes early takes the next unit)
    const int variant = (h->ozaki_variant == 0 || h->ozaki_variant == 7) ? 0 : 1;
    const bool dyn = h->ozaki_variant >= 5;
    const int tkb = 128;
    auto up = [](size_t x, size_t a) { return (x + a - 1) / a * a; };

    // every product's K pieces: one (A, B, k), or its K-segments (CRT only), each padded to KPAD
    struct Piece {
        const double* A;
        const double* B;
        int64_t lda, ldb, k, k_off, k_pad;
    };
    std::vector<Piece> pieces;
    std::vector<int32_t> piece_begin(T + 1);
    std::vector<int64_t> k_total(T), k_pads(T);
    int64_t k_pad_max = 0;
    for (int i = 0; i < T; ++i) {
        const OzProblem& p = probs[i];
        if (!crt && (p.nseg > 0 || p.stack)) return DGT_ERROR_UNSUPPORTED;
        if (p.stack) {  // a further stack of the preceding output
            if (i == 0 || p.beta != 0.0) return fail(h, DGT_ERROR_INVALID_VALUE, "stack product without its output");
            const OzProblem& q = probs[i - 1];
            if (q.m != p.m || q.n != p.n || q.C != p.C || q.ldc != p.ldc)
                return fail(h, DGT_ERROR_INVALID_VALUE, "stack product with another output");
        }
        piece_begin[i] = (int32_t)pieces.size();
        int64_t kt = 0, kp = 0;
        const int ns = p.nseg > 0 ? p.nseg : 1;
        for (int s = 0; s < ns; ++s) {
            Piece pc = p.nseg > 0 ? Piece{p.segs[s].A, p.segs[s].B, p.segs[s].lda, p.segs[s].ldb, p.segs[s].k, 0, 0}
                                  : Piece{p.A, p.B, p.lda, p.ldb, p.k, 0, 0};
            if (pc.k <= 0) continue;
            pc.k_off = kp;
            pc.k_pad = ceil_div(pc.k, oz::KPAD) * oz::KPAD;
            kt += pc.k;
            kp += pc.k_pad;
            pieces.push_back(pc);
        }
        if (kt == 0) return fail(h, DGT_ERROR_INVALID_VALUE, "grouped product without K");
        k_total[i] = kt;
        k_pads[i] = kp;
        k_pad_max = std::max(k_pad_max, kp);
    }
    piece_begin[T] = (int32_t)pieces.size();
    const int NJ = 2 * (int)pieces.size();  // split jobs: every piece of op(A), then of op(B), per product
    std::vector<oz::Seg> segs;
    std::vector<oz::Group> groups;
    oz2::CrtConst cc;
    oz2::ModTable mt;
    if (crt) {
        // one group per modulus, each the residue product over the product's own K
        if (k_pad_max >= (int64_t)1 << 17) return DGT_ERROR_UNSUPPORTED;
        oz2::crt_constants(S, cc, mt);
        for (int j = 0; j < S; ++j) {
            segs.push_back(oz::Seg{j, j, 0, -1});
            groups.push_back(oz::Group{j, j + 1, 0, mt.p[j]});
        }
    } else {
        // The flush schedule is built for the longest K: a group that is exact for it is exact
        // for every shorter K.  Segments run over each product's own K (kb1 = -1).
        if (!ozaki_schedule(S, k_pad_max, tkb, false, segs, groups) || segs.size() > (size_t)oz::MAX_SEGS ||
            groups.size() > (size_t)oz::MAX_GROUPS)
            return DGT_ERROR_UNSUPPORTED;
        for (oz::Seg& sg : segs) {
            if (sg.kb0 != 0) return DGT_ERROR_UNSUPPORTED;  // K-chunked diagonals: not in grouped form
            sg.kb1 = -1;
        }
    }

    // Tiles are numbered product by product, longest K first, so the persistent CTAs' static
    // round-robin takes the heaviest tiles early.
    std::vector<int> order(T);
    for (int i = 0; i < T; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return k_total[a] > k_total[b]; });

    // scratch: per product planes A | planes B | residues (CRT) (1 KB aligned), then all amax
    // words, all exponents
    struct Off {
        int64_t m_pad, n_pad, k_pad;
        size_t pa, pb, rs, xa, xb, ea, eb;
        int bits;
    };
    std::vector<Off> off(T);
    size_t planes = 0, amax_words = 0, exp_words = 0;
    for (int i = 0; i < T; ++i) {
        const OzProblem& p = probs[i];
        Off& o = off[i];
        o.m_pad = ceil_div(p.m, oz::TM) * oz::TM;
        o.n_pad = ceil_div(p.n, oz::TN) * oz::TN;
        o.k_pad = k_pads[i];
        o.bits = crt ? oz2::sigma_sum_for(S, k_total[i]) : 0;  // sigma_A + sigma_B
        if ((int64_t)S * std::max(o.m_pad, o.n_pad) > INT32_MAX) return DGT_ERROR_UNSUPPORTED;
        o.pa = planes;
        planes += up((size_t)S * o.m_pad * o.k_pad, 1024);
        o.pb = planes;
        planes += up((size_t)S * o.n_pad * o.k_pad, 1024);
        o.rs = planes;
        if (crt) planes += up((size_t)S * o.m_pad * o.n_pad, 1024);
        o.xa = amax_words;
        amax_words += (size_t)p.m;
        o.xb = amax_words;
        amax_words += (size_t)p.n;
        o.ea = exp_words;
        exp_words += (size_t)p.m;
        o.eb = exp_words;
        exp_words += (size_t)p.n;
    }
    // CRT: the rows' integer 2-norm bounds follow the amax words
    const size_t amax_at = planes, exp_at = up(amax_at + amax_words * 8 * (crt ? 2 : 1), 256);
    const size_t sched_at = up(exp_at + exp_words * 4, 256);  // the GEMM's unit counter (dynamic order)
    const size_t total = sched_at + 256;
    void* ws = nullptr;
    dgt_status st = ensure_workspace(h, total, &ws, 0);
    if (st != DGT_SUCCESS) return st;
    char* base = (char*)ws;
    auto* amax = (unsigned long long*)(base + amax_at);
    auto* exps = (int32_t*)(base + exp_at);
    auto* sched = (int32_t*)(base + sched_at);

    // host tables: GProb[T] (tensor maps inside, 64-byte aligned), SplitJob[NJ] and, for CRT,
    // CrtJob[T], zeroed byte for byte so that padding hashes the same on every call
    const size_t job_bytes = (size_t)NJ * sizeof(oz::SplitJob);
    const size_t crt_bytes = crt ? (size_t)T * sizeof(oz2::CrtJob) : 0;
    static thread_local std::vector<oz::GProb> host_gp;
    static thread_local std::vector<oz::SplitJob> host_jobs;
    static thread_local std::vector<oz2::CrtJob> host_crt;
    host_gp.resize(T);
    host_jobs.resize((size_t)NJ);
    host_crt.resize(crt ? T : 1);
    std::memset((void*)host_gp.data(), 0, (size_t)T * sizeof(oz::GProb));
    std::memset((void*)host_jobs.data(), 0, job_bytes);
    std::memset((void*)host_crt.data(), 0, host_crt.size() * sizeof(oz2::CrtJob));
    oz::GProb* gp = host_gp.data();
    oz::SplitJob* jobs = host_jobs.data();
    oz2::CrtJob* cj = host_crt.data();
    int64_t amax_blocks = 0, split_blocks = 0, crt_threads = 0;
    int32_t tiles = 0;
    int nj = 0;
    for (int r = 0; r < T; ++r) {
        const int i = order[r];
        const OzProblem& p = probs[i];
        const Off& o = off[i];
        void* pA = base + o.pa;
        void* pB = base + o.pb;
        oz::GProb& g = gp[r];
        if (!oz::make_plane_map(&g.tmA, pA, (int64_t)S * o.m_pad, o.k_pad, oz::TM, tkb) ||
            !oz::make_plane_map(&g.tmB, pB, (int64_t)S * o.n_pad, o.k_pad, oz::TN, tkb))
            return fail(h, DGT_ERROR_CUDA, "cuTensorMapEncodeTiled failed");
        g.m = p.m;
        g.n = p.n;
        g.ldc = p.ldc;
        g.C = p.C;
        g.row_exp = exps + o.ea;
        g.col_exp = exps + o.eb;
        g.alpha = p.alpha;
        g.beta = p.beta;
        g.m_pad = (int32_t)o.m_pad;
        g.n_pad = (int32_t)o.n_pad;
        g.nkb = (int32_t)(o.k_pad / tkb);
        g.tiles_m = (int32_t)(o.m_pad / oz::TM);
        g.tiles_n = (int32_t)(o.n_pad / oz::TN);
        g.tile_begin = tiles;
        if (crt) {
            g.res = (uint8_t*)(base + o.rs);
            g.res_ld = o.m_pad;
            g.res_plane = o.m_pad * o.n_pad;
        }
        tiles += g.tiles_m * g.tiles_n;
        // op(A) is m x k: 'N' -> MN-contiguous; op(B) as its transpose n x k: 'N' -> K-contiguous
        const bool kc[2] = {p.ta, !p.tb};
        const int64_t MN[2] = {p.m, p.n}, pad[2] = {o.m_pad, o.n_pad};
        const size_t xo[2] = {o.xa, o.xb}, eo[2] = {o.ea, o.eb};
        char* pl[2] = {(char*)pA, (char*)pB};
        for (int t = 0; t < 2; ++t) {
            for (int pi = piece_begin[i]; pi < piece_begin[i + 1]; ++pi) {
                const Piece& pc = pieces[pi];
                oz::SplitJob& J = jobs[nj++];
                J.X = t == 0 ? pc.A : pc.B;
                J.ld = t == 0 ? pc.lda : pc.ldb;
                J.MN = MN[t];
                J.K = pc.k;
                J.mn_pad = pad[t];
                J.k_pad = pc.k_pad;
                J.plane_ld = o.k_pad;
                J.amax = amax + xo[t];
                J.qn = crt ? amax + amax_words + xo[t] : nullptr;
                J.exps = exps + eo[t];
                J.planes = pl[t] + pc.k_off;  // the piece's first column of every plane row
                J.kcontig = kc[t] ? 1 : 0;
                J.amax_bx = (int32_t)(kc[t] ? ceil_div(MN[t], 8) : ceil_div(MN[t], 256));
                J.amax_by = (int32_t)(kc[t] ? 1 : ceil_div(pc.k, oz::AMAX_KCHUNK));
                J.split_bx = (int32_t)ceil_div(pad[t], crt ? oz2::RES_ROWS : 128);
                J.amax_begin = amax_blocks;
                J.split_begin = split_blocks;
                J.bits = t == 0 ? (o.bits + 1) / 2 : o.bits / 2;  // op(A) takes the odd bit
                amax_blocks += (int64_t)J.amax_bx * J.amax_by;
                split_blocks += (int64_t)J.split_bx * (pc.k_pad / (crt ? oz2::RES_KSPAN : 32));
            }
        }
    }
    // reconstruction jobs in the caller's order, so a stack group's members follow its lead
    int lead = -1;
    for (int i = 0; crt && i < T; ++i) {
        const OzProblem& p = probs[i];
        const Off& o = off[i];
        oz2::CrtJob& c = cj[i];
        c.res = (const uint8_t*)(base + o.rs);
        c.res_ld = o.m_pad;
        c.res_plane = o.m_pad * o.n_pad;
        c.m = p.m;
        c.n = p.n;
        c.row_exp = exps + o.ea;
        c.col_exp = exps + o.eb;
        c.alpha = p.alpha;
        c.beta = p.beta;
        c.C = p.C;
        c.ldc = p.ldc;
        c.bits = o.bits;  // the reconstruction's shift takes the sum
        c.thread_begin = crt_threads;
        if (p.stack) {
            cj[lead].count += 1;  // owns no threads: thread_begin is the next lead's
        } else {
            lead = i;
            c.count = 1;
            crt_threads += ceil_div(p.m, 4) * p.n;
        }
    }
    if (amax_blocks > INT32_MAX || split_blocks > INT32_MAX || crt_threads / 256 > INT32_MAX)
        return fail(h, DGT_ERROR_UNSUPPORTED, "grouped Ozaki batch too large for one launch");

    // device copy of the tables from the handle's cache (a repeated call, e.g. from a
    // replayed CUDA graph, needs no copy)
    static thread_local std::vector<int32_t> host_tiles;
    host_tiles.resize(T);
    for (int r = 0; r < T; ++r) host_tiles[r] = gp[r].tile_begin;
    const void* parts[4] = {gp, jobs, host_tiles.data(), cj};
    const size_t part_bytes[4] = {(size_t)T * sizeof(oz::GProb), job_bytes, (size_t)T * sizeof(int32_t), crt_bytes};
    size_t offs[4];
    void* table = nullptr;
    st = device_table(h, crt ? 4 : 3, parts, part_bytes, &table, offs);
    if (st != DGT_SUCCESS) return st;
    cudaStream_t s = h->stream;
    const auto* d_gp = (const oz::GProb*)((char*)table + offs[0]);
    const auto* d_jobs = (const oz::SplitJob*)((char*)table + offs[1]);
    const auto* d_tiles = (const int32_t*)((char*)table + offs[2]);
    const auto* d_crt = crt ? (const oz2::CrtJob*)((char*)table + offs[3]) : nullptr;

    mark(h, 0);
    DGT_CUDA_TRY(h, cudaMemsetAsync(amax, 0, amax_words * 8 * (crt ? 2 : 1), s));
    oz::amax_grouped<<<(unsigned)amax_blocks, 256, 0, s>>>(d_jobs, NJ);
    h->launches.fetch_add(1);
    DGT_CUDA_TRY(h, cudaGetLastError());
    if (crt) {
        DGT_CUDA_TRY(h, oz2::launch_qnorm_grouped(s, d_jobs, NJ, amax_blocks));
        h->launches.fetch_add(1);
        DGT_CUDA_TRY(h, oz2::launch_split_residues_grouped(s, d_jobs, NJ, split_blocks, S, mt));
    } else {
        oz::split_grouped<<<(unsigned)split_blocks, 128, 0, s>>>(d_jobs, NJ, S);
        DGT_CUDA_TRY(h, cudaGetLastError());
    }
    h->launches.fetch_add(1);

    static thread_local oz::Params prm;
    prm = oz::Params{};
    prm.ngroups = (int32_t)groups.size();
    std::copy(segs.begin(), segs.end(), prm.segs);
    std::copy(groups.begin(), groups.end(), prm.groups);
    prm.segs_ext = nullptr;
    prm.groups_ext = nullptr;
    prm.err = h->dev_error;
    prm.test_stall = h->test_stall == 1 ? 1 : 0;
    prm.gprobs = d_gp;
    prm.prob_tiles = d_tiles;
    prm.nprob = T;
    prm.total_tiles = tiles;
    if (dyn) {
        DGT_CUDA_TRY(h, cudaMemsetAsync(sched, 0, sizeof(int32_t), s));
        prm.sched = sched;
    }
    // the residue epilogue works in (tile, modulus) units: as many CTAs as units, up to the SMs
    const int64_t units = crt ? (int64_t)tiles * (int64_t)groups.size() : (int64_t)tiles;
    const int grid = (int)std::min<int64_t>(units, h->num_sms);
    mark(h, 1);
    cudaError_t le;
    if (crt)
        le = variant == 0 ? launch_ozaki_grouped<oz::OzCfg<4, 128, 4>, 2>(prm, grid, s)
                          : launch_ozaki_grouped<oz::OzCfg<8, 128, 4>, 2>(prm, grid, s);
    else
        le = variant == 0 ? launch_ozaki_grouped<oz::OzCfg<4, 128, 4>, 0>(prm, grid, s)
                          : launch_ozaki_grouped<oz::OzCfg<8, 128, 4>, 0>(prm, grid, s);
    h->launches.fetch_add(1);
    if (le != cudaSuccess) return cuda_fail(h, le, "grouped digit GEMM launch");
    mark(h, 2);
    if (crt) {
        DGT_CUDA_TRY(h, oz2::launch_crt_grouped(s, d_crt, T, crt_threads, cc, S));
        h->launches.fetch_add(1);
    }
    return DGT_SUCCESS;
}

dgt_status ozaki_amax(dgt_context* h, cudaStream_t s, const double* X, int64_t ld, int64_t MN, int64_t K,
                      bool kcontig, unsigned long long* out) {
    if (kcontig) {
        oz::amax_k_contig<<<(unsigned)ceil_div(MN, 8), 256, 0, s>>>(X, ld, MN, K, out);
    } else {
        DGT_CUDA_TRY(h, cudaMemsetAsync(out, 0, (size_t)MN * 8, s));
        dim3 grid((unsigned)ceil_div(MN, 256), (unsigned)ceil_div(K, oz::AMAX_KCHUNK));
        oz::amax_mn_contig<<<grid, 256, 0, s>>>(X, ld, MN, K, oz::AMAX_KCHUNK, out);
    }
    if (h) h->launches.fetch_add(1);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DGT_SUCCESS : cuda_fail(h, e, "ozaki amax");
}

}  // namespace dgt
