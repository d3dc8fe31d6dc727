// Native FP64 GEMM on the FP64 tensor cores of sm_100a (DMMA, mma.sync .f64).
//
// This is the drop-in for the reference's local cublasDgemm (src/25DCannon.cpp:324-325,
// :356-357; src/25DCannonNCCL.cpp:165-166, :202-203, :260-261, :291-292).  tcgen05 has no
// FP64 kind, so FP64 tensor work on Blackwell goes through warp-level DMMA.
//
// One persistent kernel serves every caller: a plain GEMM is one problem with one
// K-segment; a SUMMA / Cannon virtual rank is one problem whose K-segments are its step
// schedule (panel reads replace the reference's broadcasts and shifts); a grouped
// workload is many problems.  CTAs walk a static round-robin tile list.  The one inter-CTA
// wait is the 2.5D stack reduction's: a stack-0 tile waits for partial tiles numbered before
// it, the launch is cooperative (every CTA resident), so the lowest unfinished tile can always
// proceed; the wait is bounded all the same.
//
// Tile: 128 x 128 x 16, 8 warps (2 x 4), warp tile 64 x 32 of m16n8k4 DMMAs, a 4-stage
// cp.async ring in shared memory padded so fragment loads are bank-conflict free.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "dgt_internal.cuh"
#include "tc_engine.cuh"

namespace dgt {
namespace {

constexpr int BM = 128, BN = 128;
constexpr int PAD = 4;
constexpr int LD_MN = BM + PAD;  // [k][mn] layout row stride (doubles): 1056 B = 32 mod 128 banks
constexpr int GROUP_M = 8;       // tile rasterisation group for L2 reuse

// Kernel variants (the autotuner's knob): DMMA shape m16n8k{4,8,16}, K depth of a stage, ring depth.
//
// PERM (k8 / k16 shapes only): fragments are read with 128-bit shared loads.  MMA rows g
// and g+8 of an m16 tile are taken from adjacent physical rows 2g and 2g+1, and inside
// every 8-deep K block logical k = t + 4h is read from physical k = 2t + h (h = 0, 1), the
// same for A and B, so the product is unchanged.  Paddings keep every 8-lane phase of
// those loads on distinct banks: [k][mn] rows of 130 doubles (1040 B = 16 mod 128),
// A's [mn][k] rows of BK+4, B's [n][k] rows of BK+8 doubles (32 and 64 mod 128 B).
template <int MMAK_, int BK_, int STAGES_, int NWARPS_ = 8, bool PERM_ = false>
struct Cfg {
    static constexpr int MMAK = MMAK_, BK = BK_, STAGES = STAGES_;
    static constexpr bool PERM = PERM_;
    static constexpr int THREADS = NWARPS_ * 32;
    static constexpr int WARPS_M = NWARPS_ / 4;      // warps along M (4 along N, 32 columns each)
    static constexpr int MT = BM / WARPS_M / 16;     // m16 tiles per warp
    static constexpr int LDMN = PERM ? BM + 2 : LD_MN;  // [k][mn] row stride (doubles)
    static constexpr int LD_K = BK + PAD;  // [mn][k] row stride: (BK+4)*8 B = 32 mod 128 for BK in {16, 32}
    static constexpr int LD_KB = PERM ? BK + 8 : LD_K;  // B's [n][k] row stride
    static constexpr int STAGE_A = (BM * LD_K > BK * LDMN) ? BM * LD_K : BK * LDMN;
    static constexpr int STAGE_B = (BN * LD_KB > BK * LDMN) ? BN * LD_KB : BK * LDMN;
    static constexpr size_t SMEM = (size_t)STAGES * (STAGE_A + STAGE_B) * sizeof(double);
};
constexpr int MAX_INLINE_PROBS = 32, MAX_INLINE_SEGS = 160;

struct GroupedParams {
    int nprob;
    int total_tiles;
    const Problem* probs;  // global table, or null -> inline
    const KSegment* segs;
    int32_t* red_flags;    // stack-reduction counters (null: no problem reduces)
    unsigned int* err;     // sticky device error word
    int32_t test_stall;    // DGT_TUNE_TEST_STALL: 1 withholds the first stage (decoupled kernel),
                           // 2 keeps partial tiles from counting themselves
    Problem inl_probs[MAX_INLINE_PROBS];
    KSegment inl_segs[MAX_INLINE_SEGS];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// m16n8k16 (sm_90+ shape): A fragment a[2h] = A[g][t + 4h], a[2h+1] = A[g + 8][t + 4h],
// B fragment b[h] = B[t + 4h][g], h = 0..3 (the k8 layout extended along K).
__device__ __forceinline__ void dmma_16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
        "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
          "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// Loads one BK-slice of an operand tile into shared memory.
//  mn_major: global element (mn, k) at base[mn + k*ld]  -> smem [k][mn], row stride LD_MN
//  else    : global element (mn, k) at base[k + mn*ld]  -> smem [mn][k], row stride LD_K
// mn_lim / k_lim: valid extents from (mn0, k0); outside is zero-filled.
template <int BK, int LD_K, int THREADS, int LD_MN = dgt::LD_MN>
__device__ __forceinline__ void load_tile(double* s, const double* base, int64_t ld, bool mn_major, int64_t mn0,
                                          int64_t k0, int64_t mn_lim, int64_t k_lim, bool vec16, int tid) {
    const uint32_t s_base = smem_u32(s);
    if (mn_major) {
        // BK columns of BM contiguous doubles: BK*64 two-double chunks
#pragma unroll
        for (int i = 0; i < BK * 64 / THREADS; ++i) {
            int c = tid + i * THREADS;
            int k = c >> 6;
            int mn = (c & 63) * 2;
            int64_t rem = mn_lim - mn;
            int valid = (k < k_lim) ? (int)(rem >= 2 ? 2 : (rem > 0 ? rem : 0)) : 0;
            const double* src = valid ? base + (mn0 + mn) + (k0 + k) * ld : base;
            uint32_t dst = s_base + (uint32_t)((k * LD_MN + mn) * 8);
            if (vec16) {
                cp_async16(dst, src, valid * 8);
            } else {
                cp_async8(dst, src, valid >= 1 ? 8 : 0);
                const double* src1 = valid >= 2 ? src + 1 : base;
                cp_async8(dst + 8, src1, valid >= 2 ? 8 : 0);
            }
        }
    } else {
        // BM rows of BK contiguous doubles: BM*BK/2 two-double chunks
#pragma unroll
        for (int i = 0; i < BM * BK / 2 / THREADS; ++i) {
            int c = tid + i * THREADS;
            int mn = c / (BK / 2);
            int k = (c % (BK / 2)) * 2;
            int64_t rem = k_lim - k;
            int valid = (mn < mn_lim) ? (int)(rem >= 2 ? 2 : (rem > 0 ? rem : 0)) : 0;
            const double* src = valid ? base + (k0 + k) + (mn0 + mn) * ld : base;
            uint32_t dst = s_base + (uint32_t)((mn * LD_K + k) * 8);
            if (vec16) {
                cp_async16(dst, src, valid * 8);
            } else {
                cp_async8(dst, src, valid >= 1 ? 8 : 0);
                const double* src1 = valid >= 2 ? src + 1 : base;
                cp_async8(dst + 8, src1, valid >= 2 ? 8 : 0);
            }
        }
    }
}

// Interior fast path of load_tile: every chunk in range and 16-byte aligned, so each thread
// walks one base pointer with a constant stride and no per-chunk checks.
template <int BK, int LD_K, int THREADS, int LD_MN>
__device__ __forceinline__ void load_tile_full(double* s, const double* base, int64_t ld, bool mn_major, int64_t mn0,
                                               int64_t k0, int tid) {
    const uint32_t s_base = smem_u32(s);
    if (mn_major) {
        constexpr int KSTEP = THREADS / 64;  // k rows covered by one pass of the block
        const int mn = (tid & 63) * 2, kb = tid / 64;
        const double* src = base + (mn0 + mn) + (k0 + kb) * ld;
        const int64_t step = (int64_t)KSTEP * ld;
        const uint32_t dst = s_base + (uint32_t)((kb * LD_MN + mn) * 8);
#pragma unroll
        for (int i = 0; i < BK / KSTEP; ++i) cp_async16(dst + (uint32_t)(i * KSTEP * LD_MN * 8), src + i * step, 16);
    } else {
        constexpr int HB = BK / 2, MSTEP = THREADS / HB;  // rows covered by one pass of the block
        const int mn = tid / HB, k = (tid % HB) * 2;
        const double* src = base + (k0 + k) + (mn0 + mn) * ld;
        const int64_t step = (int64_t)MSTEP * ld;
        const uint32_t dst = s_base + (uint32_t)((mn * LD_K + k) * 8);
#pragma unroll
        for (int i = 0; i < BM / MSTEP; ++i) cp_async16(dst + (uint32_t)(i * MSTEP * LD_K * 8), src + i * step, 16);
    }
}

__device__ __forceinline__ int32_t ld_acquire_gpu(const int32_t* p) {
    int32_t v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add_gpu(int32_t* p, int32_t v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int find_problem(const Problem* P, int nprob, int tile) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (P[mid].tile_begin <= tile)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// One BK-deep k-tile of the CTA tile from shared memory: every warp multiplies its 64 x 32
// (or 32 x 32) block with DMMA fragments read from the stage (layouts as in load_tile).
template <class CF>
__device__ __forceinline__ void mma_ktile(const double* __restrict__ a, const double* __restrict__ b, bool a_mn,
                                          bool b_mn, double (&acc)[CF::MT][4][4], int wm, int wn, int g, int t) {
    constexpr int BK = CF::BK, LD_K = CF::LD_K, LD_KB = CF::LD_KB, LDMN = CF::LDMN;
    constexpr int MMAK = CF::MMAK, MT = CF::MT, WTM = MT * 16;
    constexpr bool PERM = CF::PERM;
    if constexpr (PERM) {
        // physical k of fragment element h (logical k = t + 4h), see Cfg
        auto kp = [&](int h) { return 8 * (h >> 1) + 2 * t + (h & 1); };
#pragma unroll
        for (int kk = 0; kk < BK; kk += MMAK) {
            double bf[4][MMAK / 4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int n = wn * 32 + j * 8 + g;
                if (b_mn) {
#pragma unroll
                    for (int h = 0; h < MMAK / 4; ++h) bf[j][h] = b[(kk + kp(h)) * LDMN + n];
                } else {
#pragma unroll
                    for (int q = 0; q < MMAK / 8; ++q) {
                        const double2 v = *reinterpret_cast<const double2*>(b + n * LD_KB + kk + 8 * q + 2 * t);
                        bf[j][2 * q] = v.x;
                        bf[j][2 * q + 1] = v.y;
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const int mr = wm * WTM + i * 16 + 2 * g;  // physical rows of MMA rows g, g + 8
                double af[MMAK / 2];
                if (a_mn) {
#pragma unroll
                    for (int h = 0; h < MMAK / 4; ++h) {
                        const double2 v = *reinterpret_cast<const double2*>(a + (kk + kp(h)) * LDMN + mr);
                        af[2 * h] = v.x;
                        af[2 * h + 1] = v.y;
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < MMAK / 8; ++q) {
                        const double2 v0 = *reinterpret_cast<const double2*>(a + mr * LD_K + kk + 8 * q + 2 * t);
                        const double2 v1 =
                            *reinterpret_cast<const double2*>(a + (mr + 1) * LD_K + kk + 8 * q + 2 * t);
                        af[4 * q] = v0.x;
                        af[4 * q + 1] = v1.x;
                        af[4 * q + 2] = v0.y;
                        af[4 * q + 3] = v1.y;
                    }
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if constexpr (MMAK == 8)
                        dmma_16x8x8(acc[i][j], af, bf[j]);
                    else
                        dmma_16x8x16(acc[i][j], af, bf[j]);
                }
            }
        }
    } else {
#pragma unroll
    for (int kk = 0; kk < BK; kk += MMAK) {
        // B fragments of the warp's four n8 tiles, then one m16 tile of A at a time
        double bf[4][MMAK / 4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = wn * 32 + j * 8 + g;
#pragma unroll
            for (int h = 0; h < MMAK / 4; ++h)
                bf[j][h] = b_mn ? b[(kk + t + 4 * h) * LDMN + n] : b[n * LD_KB + kk + t + 4 * h];
        }
#pragma unroll
        for (int i = 0; i < MT; ++i) {
            const int m = wm * WTM + i * 16 + g;
            double af[MMAK / 2];
#pragma unroll
            for (int h = 0; h < MMAK / 4; ++h) {
                if (a_mn) {
                    af[2 * h] = a[(kk + t + 4 * h) * LDMN + m];
                    af[2 * h + 1] = a[(kk + t + 4 * h) * LDMN + m + 8];
                } else {
                    af[2 * h] = a[m * LD_K + kk + t + 4 * h];
                    af[2 * h + 1] = a[(m + 8) * LD_K + kk + t + 4 * h];
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if constexpr (MMAK == 4) {
                    dmma_16x8x4(acc[i][j], af[0], af[1], bf[j][0]);
                } else if constexpr (MMAK == 8) {
                    dmma_16x8x8(acc[i][j], af, bf[j]);
                } else {
                    dmma_16x8x16(acc[i][j], af, bf[j]);
                }
            }
        }
    }
    }  // PERM
}

// C = alpha acc + beta C for the warp's fragment of tile (m0, n0) (beta == 0: C is not read).
// With nred > 0 the nred partial tiles red + s * red_stride (leading dimension red_ld) are
// added to the result afterwards, in order s = 0, 1, ... (the stack reduction's order); they were
// written by other CTAs of this launch, so they are read from L2.
template <class CF>
__device__ __forceinline__ void store_tile(const double (&acc)[CF::MT][4][4], double* C, int64_t ldc, int64_t m,
                                           int64_t n, int64_t m0, int64_t n0, double alpha, double beta, int wm,
                                           int wn, int g, int t, const double* red = nullptr,
                                           int64_t red_stride = 0, int64_t red_ld = 0, int nred = 0) {
    constexpr int MT = CF::MT, WTM = MT * 16;
    constexpr bool PERM = CF::PERM;
#pragma unroll
    for (int i = 0; i < MT; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                int64_t row = m0 + wm * WTM + i * 16 + (PERM ? 2 * g + h : g + h * 8);
                if (row >= m) continue;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    int64_t col = n0 + wn * 32 + j * 8 + 2 * t + e;
                    if (col >= n) continue;
                    double* cp = C + row + col * ldc;
                    double v = alpha * acc[i][j][h * 2 + e];
                    if (beta != 0.0) v = fma(beta, *cp, v);
                    // explicit adds: alpha acc + partial must not contract into one FMA
                    for (int s = 0; s < nred; ++s) v = __dadd_rn(v, __ldcg(red + s * red_stride + row + col * red_ld));
                    *cp = v;
                }
            }
        }
    }
}

template <class CF>
__global__ void __launch_bounds__(CF::THREADS, 1) dmma_grouped_kernel(const __grid_constant__ GroupedParams prm) {
    constexpr int BK = CF::BK, STAGES = CF::STAGES, LD_K = CF::LD_K, LD_KB = CF::LD_KB, LDMN = CF::LDMN;
    constexpr int STAGE_A = CF::STAGE_A, STAGE_B = CF::STAGE_B;
    constexpr int THREADS = CF::THREADS, MT = CF::MT;
    static_assert(!CF::PERM || CF::MMAK >= 8, "128-bit fragment loads need the k8 or k16 shape");
    extern __shared__ __align__(16) double smem[];
    double* sA = smem;
    double* sB = smem + STAGES * STAGE_A;

    const Problem* probs = prm.probs ? prm.probs : prm.inl_probs;
    const KSegment* segs = prm.segs ? prm.segs : prm.inl_segs;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 2, wn = warp & 3;  // WARPS_M x 4 warps
    const int g = lane >> 2, t = lane & 3;

    for (int tile = blockIdx.x; tile < prm.total_tiles; tile += gridDim.x) {
        const int pi = find_problem(probs, prm.nprob, tile);
        const Problem pb = probs[pi];
        // grouped rasterisation inside the problem
        int local = tile - pb.tile_begin;
        int in_group = GROUP_M * pb.tiles_n;
        int group = local / in_group;
        int first_m = group * GROUP_M;
        int gsize = min(pb.tiles_m - first_m, GROUP_M);
        int tm = first_m + (local % in_group) % gsize;
        int tn = (local % in_group) / gsize;
        const int64_t m0 = (int64_t)tm * BM, n0 = (int64_t)tn * BN;
        const bool a_mn = (pb.transa == 0);  // A 'N': element (m,k) at A[m + k*lda]
        const bool b_mn = (pb.transb != 0);  // B 'T': element (n,k) at B[n + k*ldb]

        int total_kt = 0;
        for (int s = 0; s < pb.seg_count; ++s) total_kt += (int)ceil_div(segs[pb.seg_begin + s].k, BK);

        double acc[MT][4][4];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

        // loader state: which segment / k offset the next k-tile comes from
        int ld_seg = 0;
        int64_t ld_k0 = 0;
        int issued = 0;
        auto issue = [&](int stage) {
            if (issued < total_kt) {
                while (segs[pb.seg_begin + ld_seg].k <= 0) ++ld_seg;  // skip empty segments
                const KSegment sg = segs[pb.seg_begin + ld_seg];
                int64_t klim = sg.k - ld_k0;
                bool va = (((uintptr_t)sg.A & 15) == 0) && ((sg.lda & 1) == 0);
                bool vb = (((uintptr_t)sg.B & 15) == 0) && ((sg.ldb & 1) == 0);
                if (va && klim >= BK && pb.m - m0 >= BM)
                    load_tile_full<BK, LD_K, THREADS, LDMN>(sA + stage * STAGE_A, sg.A, sg.lda, a_mn, m0, ld_k0, tid);
                else
                    load_tile<BK, LD_K, THREADS, LDMN>(sA + stage * STAGE_A, sg.A, sg.lda, a_mn, m0, ld_k0, pb.m - m0,
                                                       klim, va, tid);
                if (vb && klim >= BK && pb.n - n0 >= BN)
                    load_tile_full<BK, LD_KB, THREADS, LDMN>(sB + stage * STAGE_B, sg.B, sg.ldb, b_mn, n0, ld_k0, tid);
                else
                    load_tile<BK, LD_KB, THREADS, LDMN>(sB + stage * STAGE_B, sg.B, sg.ldb, b_mn, n0, ld_k0, pb.n - n0,
                                                        klim, vb, tid);
                ld_k0 += BK;
                if (ld_k0 >= sg.k) {
                    ld_k0 = 0;
                    ++ld_seg;
                }
                ++issued;
            }
            cp_async_commit();
        };

#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s) issue(s);

        for (int kt = 0; kt < total_kt; ++kt) {
            cp_async_wait<STAGES - 2>();
            __syncthreads();
            issue((kt + STAGES - 1) % STAGES);
            const double* a = sA + (kt % STAGES) * STAGE_A;
            const double* b = sB + (kt % STAGES) * STAGE_B;
            mma_ktile<CF>(a, b, a_mn, b_mn, acc, wm, wn, g, t);
        }
        cp_async_wait<0>();
        __syncthreads();  // the next tile's prologue reuses the ring

        // epilogue: C = alpha*acc + beta*C (beta == 0: C not read), plus the stack partials
        int nred = 0;
        if (pb.red_role == 2) {
            // a stack-0 tile: its partial tiles come from CTAs that took them earlier in the
            // tile order; one thread waits (bounded) for their count, then the CTA reads them
            __shared__ int s_ready;
            if (tid == 0) {
                const int32_t* f = prm.red_flags + pb.red_slot + local;
                const long long t0 = clock64();
                int ready = 1;
                while (ld_acquire_gpu(f) < pb.red_wait) {
                    // a wait that already ran out anywhere in the launch ends this one too, so
                    // the whole launch spends one budget, not one per stack-0 tile
                    if (clock64() - t0 > oz::WAIT_BUDGET || (*(volatile unsigned int*)prm.err & DGT_DEVERR_TIMEOUT)) {
                        atomicOr(prm.err, DGT_DEVERR_TIMEOUT);
                        ready = 0;
                        break;
                    }
                    __nanosleep(256);
                }
                s_ready = ready;
            }
            __syncthreads();
            nred = s_ready ? pb.red_wait : 0;
        }
        store_tile<CF>(acc, pb.C, pb.ldc, pb.m, pb.n, m0, n0, pb.alpha, pb.beta, wm, wn, g, t, pb.red_src,
                       pb.red_stride, pb.red_ld, nred);
        if (pb.red_role == 1) {
            // a partial tile: every thread's stores reach L2 before the tile is counted
            __threadfence();
            __syncthreads();
            if (tid == 0 && prm.test_stall != 2) red_release_add_gpu(prm.red_flags + pb.red_slot + local, 1);
        }
    }
}

// ---- the grouped kernel without CTA barriers in its main loop -------------------------------
// cp.async copies signal a stage's full mbarrier when they land (cp.async.mbarrier.arrive.noinc,
// one arrival per thread), every warp releases the stage through its empty mbarrier after its
// DMMAs, and every thread refills a stage (its share of the copies) once lane 0 of its warp saw
// the stage released.  The load cursor (tile, problem, K-segment, K offset; the same in every
// thread) runs across tiles, so the next tile's first stages load while this tile's last
// k-tiles multiply and its epilogue stores, and no tile starts on an empty ring.  Every wait is
// bounded; a warp that gives up leaves its k-loop, and the CTA agrees on the abort at the tile
// boundary (one __syncthreads_and per tile).  Same fragments, same k order: the results equal
// dmma_grouped_kernel's of the same shape bit for bit.
__device__ __forceinline__ void cp_async_mbar_arrive(uint32_t bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(bar) : "memory");
}

// Tile `local` of a problem: grouped rasterisation (GROUP_M tile rows at a time).
__device__ __forceinline__ void tile_origin(const Problem& pb, int local, int64_t& m0, int64_t& n0) {
    const int in_group = GROUP_M * pb.tiles_n;
    const int first_m = (local / in_group) * GROUP_M;
    const int gsize = min(pb.tiles_m - first_m, GROUP_M);
    m0 = (int64_t)(first_m + (local % in_group) % gsize) * BM;
    n0 = (int64_t)((local % in_group) / gsize) * BN;
}

template <class CF>
constexpr size_t grouped_dec_smem_bytes() {
    return CF::SMEM + (size_t)CF::STAGES * 16 + 16;  // ring, full + empty barriers, abort flag
}

template <class CF>
__global__ void __launch_bounds__(CF::THREADS, 1) dmma_grouped_dec_kernel(const __grid_constant__ GroupedParams prm) {
    constexpr int BK = CF::BK, STAGES = CF::STAGES, LD_K = CF::LD_K, LD_KB = CF::LD_KB, LDMN = CF::LDMN;
    constexpr int STAGE_A = CF::STAGE_A, STAGE_B = CF::STAGE_B;
    constexpr int THREADS = CF::THREADS, MT = CF::MT, NWARPS = THREADS / 32;
    static_assert(!CF::PERM || CF::MMAK >= 8, "128-bit fragment loads need the k8 or k16 shape");
    extern __shared__ __align__(16) double smem[];
    double* sA = smem;
    double* sB = smem + STAGES * STAGE_A;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + STAGES * STAGE_B);
    uint64_t* empty = full + STAGES;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + STAGES);
    __shared__ int s_ready;

    const Problem* probs = prm.probs ? prm.probs : prm.inl_probs;
    const KSegment* segs = prm.segs ? prm.segs : prm.inl_segs;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 2, wn = warp & 3;
    const int g = lane >> 2, t = lane & 3;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            oz::mbar_init(oz::su32(full + s), THREADS);
            oz::mbar_init(oz::su32(empty + s), NWARPS);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    // the load cursor
    int ld_tile = blockIdx.x, ld_pi = 0, ld_seg = 0;
    int64_t ld_k0 = 0, ld_m0 = 0, ld_n0 = 0;
    auto ld_enter = [&]() {  // the first non-empty K-segment of ld_tile or a later tile
        while (ld_tile < prm.total_tiles) {
            ld_pi = find_problem(probs, prm.nprob, ld_tile);
            const Problem& pb = probs[ld_pi];
            tile_origin(pb, ld_tile - pb.tile_begin, ld_m0, ld_n0);
            ld_k0 = 0;
            ld_seg = 0;
            while (ld_seg < pb.seg_count && segs[pb.seg_begin + ld_seg].k <= 0) ++ld_seg;
            if (ld_seg < pb.seg_count) return;
            ld_tile += gridDim.x;  // no K at all: its consumer multiplies nothing
        }
    };
    ld_enter();
    uint32_t issued = 0;
    // moves the cursor past the stage just issued (K offset, then segment, then tile)
    auto advance = [&](const KSegment& sg, const Problem& pb) -> bool {
        ld_k0 += BK;
        if (ld_k0 >= sg.k) {
            ld_k0 = 0;
            ++ld_seg;
            while (ld_seg < pb.seg_count && segs[pb.seg_begin + ld_seg].k <= 0) ++ld_seg;
            if (ld_seg >= pb.seg_count) {
                ld_tile += gridDim.x;
                ld_enter();
            }
        }
        return true;
    };
    // this thread's share of the next stage; false if its warp gave up waiting for the stage
    auto issue = [&]() -> bool {
        if (ld_tile >= prm.total_tiles) return true;
        const int s = (int)(issued % STAGES);
        if (issued >= STAGES) {  // the stage's previous k-tile, released by every warp
            bool good = true;
            if (lane == 0)
                good = oz::mbar_wait(oz::su32(empty + s), ((issued - STAGES) / STAGES) & 1, abort_flag, prm.err);
            if (!__shfl_sync(0xffffffffu, good, 0)) return false;
        }
        const Problem& pb = probs[ld_pi];
        const KSegment sg = segs[pb.seg_begin + ld_seg];
        const bool a_mn = (pb.transa == 0), b_mn = (pb.transb != 0);
        if (prm.test_stall == 1 && issued == 0) {  // the test hook: the first stage never fills
            ++issued;
            return advance(sg, pb);
        }
        const int64_t klim = sg.k - ld_k0;
        const bool va = (((uintptr_t)sg.A & 15) == 0) && ((sg.lda & 1) == 0);
        const bool vb = (((uintptr_t)sg.B & 15) == 0) && ((sg.ldb & 1) == 0);
        if (va && klim >= BK && pb.m - ld_m0 >= BM)
            load_tile_full<BK, LD_K, THREADS, LDMN>(sA + s * STAGE_A, sg.A, sg.lda, a_mn, ld_m0, ld_k0, tid);
        else
            load_tile<BK, LD_K, THREADS, LDMN>(sA + s * STAGE_A, sg.A, sg.lda, a_mn, ld_m0, ld_k0, pb.m - ld_m0, klim,
                                               va, tid);
        if (vb && klim >= BK && pb.n - ld_n0 >= BN)
            load_tile_full<BK, LD_KB, THREADS, LDMN>(sB + s * STAGE_B, sg.B, sg.ldb, b_mn, ld_n0, ld_k0, tid);
        else
            load_tile<BK, LD_KB, THREADS, LDMN>(sB + s * STAGE_B, sg.B, sg.ldb, b_mn, ld_n0, ld_k0, pb.n - ld_n0,
                                                klim, vb, tid);
        cp_async_mbar_arrive(oz::su32(full + s));
        ++issued;
        return advance(sg, pb);
    };

    bool ok = true;
    for (int s = 0; s < STAGES - 1 && ok; ++s) ok = issue();
    uint32_t it = 0;  // stages consumed
    for (int tile = blockIdx.x; tile < prm.total_tiles; tile += gridDim.x) {
        const int pi = find_problem(probs, prm.nprob, tile);
        const Problem& pb = probs[pi];
        const int local = tile - pb.tile_begin;
        int64_t m0, n0;
        tile_origin(pb, local, m0, n0);
        const bool a_mn = (pb.transa == 0), b_mn = (pb.transb != 0);
        int total_kt = 0;
        for (int s = 0; s < pb.seg_count; ++s) {
            const int64_t k = segs[pb.seg_begin + s].k;
            if (k > 0) total_kt += (int)ceil_div(k, BK);
        }
        double acc[MT][4][4];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
        for (int kt = 0; kt < total_kt && ok; ++kt, ++it) {
            const int s = (int)(it % STAGES);
            const bool got = oz::mbar_wait(oz::su32(full + s), (it / STAGES) & 1, abort_flag, prm.err);
            if (!__all_sync(0xffffffffu, got)) {
                ok = false;
                break;
            }
            mma_ktile<CF>(sA + s * STAGE_A, sB + s * STAGE_B, a_mn, b_mn, acc, wm, wn, g, t);
            __syncwarp();  // every lane's fragment reads of the stage are done
            if (lane == 0) oz::mbar_arrive(oz::su32(empty + s));
            if (!issue()) {
                ok = false;
                break;
            }
        }
        if (!__syncthreads_and(ok)) break;  // the CTA leaves a failed tile together

        // epilogue: as dmma_grouped_kernel's (stack partials waited for and added in order)
        int nred = 0;
        if (pb.red_role == 2) {
            if (tid == 0) {
                const int32_t* f = prm.red_flags + pb.red_slot + local;
                const long long t0 = clock64();
                int ready = 1;
                while (ld_acquire_gpu(f) < pb.red_wait) {
                    // a wait that already ran out anywhere in the launch ends this one too, so
                    // the whole launch spends one budget, not one per stack-0 tile
                    if (clock64() - t0 > oz::WAIT_BUDGET || (*(volatile unsigned int*)prm.err & DGT_DEVERR_TIMEOUT)) {
                        atomicOr(prm.err, DGT_DEVERR_TIMEOUT);
                        ready = 0;
                        break;
                    }
                    __nanosleep(256);
                }
                s_ready = ready;
            }
            __syncthreads();
            nred = s_ready ? pb.red_wait : 0;
        }
        store_tile<CF>(acc, pb.C, pb.ldc, pb.m, pb.n, m0, n0, pb.alpha, pb.beta, wm, wn, g, t, pb.red_src,
                       pb.red_stride, pb.red_ld, nred);
        if (pb.red_role == 1) {
            __threadfence();
            __syncthreads();
            if (tid == 0 && prm.test_stall != 2) red_release_add_gpu(prm.red_flags + pb.red_slot + local, 1);
        }
    }
    cp_async_wait<0>();  // this thread's copies still in flight (the lookahead past the last tile)
    __syncthreads();
}

// ---- TMA-fed form for one plain GEMM ---------------------------------------------------------
// The same CTA tile, warps and fragment code, with the operand tiles brought into shared memory
// by the tensor memory accelerator instead of per-thread cp.async: thread 0 issues two 2D
// bulk-tensor loads per stage (no multicast) that complete on the stage's mbarrier, so no
// thread spends issue slots on load addresses.  The boxes carry the padding of the cp.async
// layout: a mn-major operand box is {BM + 4, BK} (rows of 132 doubles, the extra 4 columns are
// never read) and a K-major one {BK + 4, BM}; ragged edges and the end of K come back
// zero-filled from the out-of-range part of the box.  The stage counter runs across tiles,
// so the next tile's first stages load while this tile's epilogue stores C.  Every mbarrier
// wait is bounded; on expiry the CTA records DGT_DEVERR_TIMEOUT, stops, waits (bounded) for
// its own loads and returns.
struct TmaGemmParams {
    CUtensorMap tmA, tmB;  // 64-byte aligned inside the parameter block
    int64_t m, n, ldc;
    double alpha, beta;
    double* C;
    int32_t tiles_m, tiles_n, total_tiles, ktiles;
    int32_t a_mn, b_mn;  // operand layouts: 1 = mn-major box {BM + 4, BK}, 0 = K-major box {BK + 4, BM}
    unsigned int* err;
    int32_t test_stall;  // DGT_TUNE_TEST_STALL 1: the first stage is never loaded
};

template <class CF>
__global__ void __launch_bounds__(CF::THREADS, 1) dmma_tma_kernel(const __grid_constant__ TmaGemmParams P) {
    constexpr int BK = CF::BK, STAGES = CF::STAGES, STAGE_A = CF::STAGE_A, STAGE_B = CF::STAGE_B, MT = CF::MT;
    static_assert(!CF::PERM, "the TMA boxes reproduce the unpermuted padded layouts");
    static_assert(CF::LDMN == BM + 4 && CF::LD_K == BK + 4 && CF::LD_KB == BK + 4, "box shapes follow the layouts");
    constexpr uint32_t BYTES_MN = (BM + 4) * BK * 8, BYTES_K = (BK + 4) * BM * 8;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double* smem = reinterpret_cast<double*>(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    double* sA = smem;
    double* sB = smem + STAGES * STAGE_A;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + STAGES * STAGE_B);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(full + STAGES);
    // thread 0's load cursor lives in shared memory, out of the MMA warps' registers:
    // cur[0] = tile, cur[1] = k-tile of the next stage to fill, cur[2] = stages issued
    int* cur = const_cast<int*>(abort_flag) + 1;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 2, wn = warp & 3;
    const int g = lane >> 2, t = lane & 3;
    const uint32_t tx_bytes = (P.a_mn ? BYTES_MN : BYTES_K) + (P.b_mn ? BYTES_MN : BYTES_K);

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) oz::mbar_init(oz::su32(full + s), 1);
        *abort_flag = 0;
        cur[0] = blockIdx.x;
        cur[1] = 0;
        cur[2] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    auto tile_mn = [&](int tile, int64_t& m0, int64_t& n0) {
        const int in_group = GROUP_M * P.tiles_n;
        const int first_m = (tile / in_group) * GROUP_M;
        const int gsize = min(P.tiles_m - first_m, GROUP_M);
        m0 = (int64_t)(first_m + (tile % in_group) % gsize) * BM;
        n0 = (int64_t)((tile % in_group) / gsize) * BN;
    };
    auto issue_next = [&]() {
        const int ld_tile = cur[0], ld_kt = cur[1];
        if (ld_tile >= P.total_tiles) return;
        const int s = cur[2] % STAGES;
        int64_t m0, n0;
        tile_mn(ld_tile, m0, n0);
        const int32_t k0 = ld_kt * BK;
        const uint32_t bar = oz::su32(full + s);
        if (!(P.test_stall == 1 && cur[2] == 0)) {  // (the test hook withholds the first stage)
            oz::mbar_expect_tx(bar, tx_bytes);
            const uint32_t da = oz::su32(sA + s * STAGE_A), db = oz::su32(sB + s * STAGE_B);
            if (P.a_mn)
                oz::tma_load_2d(da, &P.tmA, (int32_t)m0, k0, bar);
            else
                oz::tma_load_2d(da, &P.tmA, k0, (int32_t)m0, bar);
            if (P.b_mn)
                oz::tma_load_2d(db, &P.tmB, (int32_t)n0, k0, bar);
            else
                oz::tma_load_2d(db, &P.tmB, k0, (int32_t)n0, bar);
        }
        cur[2] += 1;
        if (ld_kt + 1 == P.ktiles) {
            cur[1] = 0;
            cur[0] = ld_tile + gridDim.x;
        } else {
            cur[1] = ld_kt + 1;
        }
    };
    if (tid == 0)
        for (int s = 0; s < STAGES - 1; ++s) issue_next();

    uint32_t it = 0;  // stages consumed
    bool ok = true;
    for (int tile = blockIdx.x; tile < P.total_tiles && ok; tile += gridDim.x) {
        int64_t m0, n0;
        tile_mn(tile, m0, n0);
        double acc[MT][4][4];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
        for (int kt = 0; kt < P.ktiles; ++kt, ++it) {
            const int s = (int)(it % STAGES);
            const bool got = oz::mbar_wait(oz::su32(full + s), (it / STAGES) & 1, abort_flag, P.err);
            // every warp is done with stage it - 1 (refilled below), and all agree on aborting
            if (__syncthreads_or(!got)) {
                ok = false;
                break;
            }
            if (tid == 0) issue_next();
            mma_ktile<CF>(sA + s * STAGE_A, sB + s * STAGE_B, P.a_mn != 0, P.b_mn != 0, acc, wm, wn, g, t);
        }
        if (!ok) break;
        store_tile<CF>(acc, P.C, P.ldc, P.m, P.n, m0, n0, P.alpha, P.beta, wm, wn, g, t);
    }
    // loads issued but not consumed (the lookahead past the last tile, or an abort) must land
    // before the CTA's shared memory is released
    if (tid == 0) {
        for (uint32_t j = it; j < (uint32_t)cur[2]; ++j) {
            if (P.test_stall == 1 && j == 0) continue;  // the withheld stage has nothing in flight
            long long t0 = clock64();
            while (!oz::mbar_try(oz::su32(full + (j % STAGES)), (j / STAGES) & 1) && clock64() - t0 < oz::WAIT_BUDGET) {
            }
        }
    }
    __syncthreads();
}

// 2D FP64 tensor map over a column-major operand: inner extent `inner` (contiguous), `outer`
// columns of stride ld doubles, box {box_inner, box_outer}, no swizzle, zero fill outside.
static bool make_f64_map(CUtensorMap* map, const double* base, int64_t inner, int64_t outer, int64_t ld,
                         int box_inner, int box_outer) {
    auto enc = oz::get_encode();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 8)};
    cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_outer};
    cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)base, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The same TMA-fed kernel without the per-k-tile __syncthreads.  Every stage has a full
// barrier (the TMA bytes land) and an empty barrier (one arrival per warp once its DMMAs have
// read the stage).  Thread 0, after consuming k-tile `it`, waits (bounded) until every warp has
// released k-tile it - 1 and refills that stage with load it + STAGES - 1; the other warps never
// wait for each other, only for data, so a warp that falls behind on one k-tile catches up on
// the next instead of holding all eight at a barrier.
// EARLY: thread 0 refills before its own DMMAs of k-tile `it` (the load goes out up to one
// k-tile sooner; warp 0 may wait for the slowest warp first).
template <class CF, bool EARLY = false>
__global__ void __launch_bounds__(CF::THREADS, 1) dmma_tma_dec_kernel(const __grid_constant__ TmaGemmParams P) {
    constexpr int BK = CF::BK, STAGES = CF::STAGES, STAGE_A = CF::STAGE_A, STAGE_B = CF::STAGE_B, MT = CF::MT;
    constexpr int NWARPS = CF::THREADS / 32;
    static_assert(!CF::PERM, "the TMA boxes reproduce the unpermuted padded layouts");
    static_assert(CF::LDMN == BM + 4 && CF::LD_K == BK + 4 && CF::LD_KB == BK + 4, "box shapes follow the layouts");
    constexpr uint32_t BYTES_MN = (BM + 4) * BK * 8, BYTES_K = (BK + 4) * BM * 8;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double* smem = reinterpret_cast<double*>(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    double* sA = smem;
    double* sB = smem + STAGES * STAGE_A;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + STAGES * STAGE_B);
    uint64_t* empty = full + STAGES;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + STAGES);
    int* cur = const_cast<int*>(abort_flag) + 1;  // thread 0's load cursor, as in dmma_tma_kernel

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 2, wn = warp & 3;
    const int g = lane >> 2, t = lane & 3;
    const uint32_t tx_bytes = (P.a_mn ? BYTES_MN : BYTES_K) + (P.b_mn ? BYTES_MN : BYTES_K);

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            oz::mbar_init(oz::su32(full + s), 1);
            oz::mbar_init(oz::su32(empty + s), NWARPS);
        }
        *abort_flag = 0;
        cur[0] = blockIdx.x;
        cur[1] = 0;
        cur[2] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    auto tile_mn = [&](int tile, int64_t& m0, int64_t& n0) {
        const int in_group = GROUP_M * P.tiles_n;
        const int first_m = (tile / in_group) * GROUP_M;
        const int gsize = min(P.tiles_m - first_m, GROUP_M);
        m0 = (int64_t)(first_m + (tile % in_group) % gsize) * BM;
        n0 = (int64_t)((tile % in_group) / gsize) * BN;
    };
    auto issue_next = [&]() {
        const int ld_tile = cur[0], ld_kt = cur[1];
        if (ld_tile >= P.total_tiles) return;
        const int s = cur[2] % STAGES;
        int64_t m0, n0;
        tile_mn(ld_tile, m0, n0);
        const int32_t k0 = ld_kt * BK;
        const uint32_t bar = oz::su32(full + s);
        if (!(P.test_stall == 1 && cur[2] == 0)) {  // (the test hook withholds the first stage)
            oz::mbar_expect_tx(bar, tx_bytes);
            const uint32_t da = oz::su32(sA + s * STAGE_A), db = oz::su32(sB + s * STAGE_B);
            if (P.a_mn)
                oz::tma_load_2d(da, &P.tmA, (int32_t)m0, k0, bar);
            else
                oz::tma_load_2d(da, &P.tmA, k0, (int32_t)m0, bar);
            if (P.b_mn)
                oz::tma_load_2d(db, &P.tmB, (int32_t)n0, k0, bar);
            else
                oz::tma_load_2d(db, &P.tmB, k0, (int32_t)n0, bar);
        }
        cur[2] += 1;
        if (ld_kt + 1 == P.ktiles) {
            cur[1] = 0;
            cur[0] = ld_tile + gridDim.x;
        } else {
            cur[1] = ld_kt + 1;
        }
    };
    if (tid == 0)
        for (int s = 0; s < STAGES - 1; ++s) issue_next();

    uint32_t it = 0;  // stages consumed by this warp
    bool ok = true;
    for (int tile = blockIdx.x; tile < P.total_tiles && ok; tile += gridDim.x) {
        int64_t m0, n0;
        tile_mn(tile, m0, n0);
        double acc[MT][4][4];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
        for (int kt = 0; kt < P.ktiles; ++kt, ++it) {
            const int s = (int)(it % STAGES);
            // every lane waits (bounded); the warp leaves together if any lane gave up
            const bool got = oz::mbar_wait(oz::su32(full + s), (it / STAGES) & 1, abort_flag, P.err);
            if (!__all_sync(0xffffffffu, got)) {
                ok = false;
                break;
            }
            // thread 0 refills the stage of k-tile it - 1 once every warp has released it
            auto refill = [&]() -> bool {
                bool good = true;
                if (lane == 0) {
                    if (it > 0) {
                        const uint32_t prev = it - 1;
                        good = oz::mbar_wait(oz::su32(empty + prev % STAGES), (prev / STAGES) & 1, abort_flag, P.err);
                    }
                    if (good) issue_next();
                }
                return __shfl_sync(0xffffffffu, good, 0);
            };
            if (EARLY && warp == 0 && !refill()) {
                ok = false;
                break;
            }
            mma_ktile<CF>(sA + s * STAGE_A, sB + s * STAGE_B, P.a_mn != 0, P.b_mn != 0, acc, wm, wn, g, t);
            __syncwarp();  // every lane's fragment reads of the stage are done
            if (lane == 0) oz::mbar_arrive(oz::su32(empty + s));
            if (!EARLY && warp == 0 && !refill()) {
                ok = false;
                break;
            }
        }
        if (!ok) break;
        store_tile<CF>(acc, P.C, P.ldc, P.m, P.n, m0, n0, P.alpha, P.beta, wm, wn, g, t);
    }
    // loads issued but not consumed (the lookahead past the last tile, or an abort) must land
    // before the CTA's shared memory is released
    if (tid == 0) {
        for (uint32_t j = it; j < (uint32_t)cur[2]; ++j) {
            if (P.test_stall == 1 && j == 0) continue;  // the withheld stage has nothing in flight
            long long t0 = clock64();
            while (!oz::mbar_try(oz::su32(full + (j % STAGES)), (j / STAGES) & 1) && clock64() - t0 < oz::WAIT_BUDGET) {
            }
        }
    }
    __syncthreads();
}

template <class CF>
constexpr size_t tma_dec_smem_bytes() {
    return 128 + CF::SMEM + (size_t)CF::STAGES * 16 + 32;  // ring, full + empty barriers, abort flag + cursor
}

template <class CF, bool EARLY = false>
cudaError_t launch_tma_dec_variant(const TmaGemmParams& prm, int grid, cudaStream_t stream) {
    static_assert(tma_dec_smem_bytes<CF>() <= 232448, "shared memory per CTA");
    cudaError_t e = smem_opt_in<dmma_tma_dec_kernel<CF, EARLY>>((int)tma_dec_smem_bytes<CF>());
    if (e != cudaSuccess) return e;
    dmma_tma_dec_kernel<CF, EARLY><<<grid, CF::THREADS, tma_dec_smem_bytes<CF>(), stream>>>(prm);
    return cudaGetLastError();
}

template <class CF>
constexpr size_t tma_smem_bytes() {
    return 128 + CF::SMEM + (size_t)CF::STAGES * 8 + 32;  // ring, full barriers, abort flag + cursor
}

template <class CF>
cudaError_t launch_tma_variant(const TmaGemmParams& prm, int grid, cudaStream_t stream) {
    cudaError_t e = smem_opt_in<dmma_tma_kernel<CF>>((int)tma_smem_bytes<CF>());
    if (e != cudaSuccess) return e;
    dmma_tma_kernel<CF><<<grid, CF::THREADS, tma_smem_bytes<CF>(), stream>>>(prm);
    return cudaGetLastError();
}

using V0 = Cfg<4, 16, 4>;
using V1 = Cfg<8, 16, 4>;
using V2 = Cfg<8, 32, 3>;
using V3 = Cfg<4, 32, 3>;
using V4 = Cfg<8, 16, 4, 16>;
using V5 = Cfg<8, 32, 3, 16>;
using V6 = Cfg<4, 16, 4, 16>;
using V7 = Cfg<16, 32, 3>;
using V8 = Cfg<16, 32, 3, 16>;
using V9 = Cfg<16, 16, 4>;
using V10 = Cfg<8, 16, 4, 8, true>;
using V11 = Cfg<16, 16, 4, 8, true>;
using V12 = Cfg<8, 32, 2, 8, true>;
using V13 = Cfg<16, 32, 2, 8, true>;

template <auto Kernel, int THREADS, size_t SMEM>
cudaError_t launch_grouped(const GroupedParams& prm, int grid, cudaStream_t stream, bool coop) {
    static_assert(SMEM <= 232448 - 16, "shared memory per CTA");
    cudaError_t e = smem_opt_in<Kernel>((int)SMEM);
    if (e != cudaSuccess) return e;
    if (!coop) {
        Kernel<<<grid, THREADS, SMEM, stream>>>(prm);
        return cudaGetLastError();
    }
    // a stack reduction waits across CTAs: a cooperative launch keeps them all resident
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = SMEM;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, Kernel, prm);
}

// DEC: the grouped kernel without CTA barriers in its main loop.
template <class CF, bool DEC = false>
cudaError_t launch_variant(const GroupedParams& prm, int grid, cudaStream_t stream, bool coop) {
    if constexpr (DEC)
        return launch_grouped<dmma_grouped_dec_kernel<CF>, CF::THREADS, grouped_dec_smem_bytes<CF>()>(prm, grid, stream,
                                                                                                    coop);
    else
        return launch_grouped<dmma_grouped_kernel<CF>, CF::THREADS, CF::SMEM>(prm, grid, stream, coop);
}

}  // namespace

// Variants 14-17: the TMA-fed kernel with the tile shapes of variants 2, 1, 7 and a 5-deep
// BK = 16 ring.  A call the TMA form does not cover (several problems or K-segments, operands
// not 16-byte aligned or with an odd leading dimension, or small) runs the cp.async kernel of
// the same shape instead.
using T14 = V2;
using T15 = V1;
using T16 = V7;
using T17 = Cfg<8, 16, 5>;
// Variants 18-22: the decoupled TMA kernel (empty barriers, no per-k-tile __syncthreads) with
// the tile shapes of 14, 17 and 16, a 4-deep BK = 24 ring (21), and 14's shape refilling
// before warp 0's DMMAs (22); outside the TMA form's cover, the cp.async kernel of variant 23
// (the decoupled grouped kernel of 18's shape), 17, 7, 2 and 2.  (BK = 24 is a TMA-only
// depth: its cp.async stand-in is variant 2.)
using T21 = Cfg<8, 24, 4>;
// Variants 23-25: the grouped kernel without CTA barriers in its main loop
// (dmma_grouped_dec_kernel) with the shapes of variants 2, 1 and 17; every call, grouped or
// not, runs it.

int dmma_variant_count() { return 26; }
int64_t dmma_tile_count(int64_t m, int64_t n) { return ceil_div(m, BM) * ceil_div(n, BN); }

// The TMA form for one plain GEMM, when the operands allow it; *used says whether it ran.
// DEC: the decoupled kernel (dmma_tma_dec_kernel).
template <class CF, bool DEC = false, bool EARLY = false>
static cudaError_t try_tma(dgt_context* h, const Problem& p, const KSegment& sg, int grid, bool* used) {
    *used = false;
    const bool a_mn = p.transa == 0, b_mn = p.transb != 0;
    const int64_t k = sg.k;
    if (p.m < 256 || p.n < 256 || k < 64) return cudaSuccess;
    if (((uintptr_t)sg.A & 15) || ((uintptr_t)sg.B & 15) || (sg.lda & 1) || (sg.ldb & 1)) return cudaSuccess;
    static thread_local TmaGemmParams prm;
    prm = TmaGemmParams{};
    // op(A) is m x k: 'N' -> mn-major (inner m), 'T' -> K-major (inner k); op(B)^T is n x k:
    // 'N' -> K-major (inner k), 'T' -> mn-major (inner n)
    const bool okA = a_mn ? make_f64_map(&prm.tmA, sg.A, p.m, k, sg.lda, BM + 4, CF::BK)
                          : make_f64_map(&prm.tmA, sg.A, k, p.m, sg.lda, CF::BK + 4, BM);
    const bool okB = b_mn ? make_f64_map(&prm.tmB, sg.B, p.n, k, sg.ldb, BN + 4, CF::BK)
                          : make_f64_map(&prm.tmB, sg.B, k, p.n, sg.ldb, CF::BK + 4, BN);
    if (!okA || !okB) return cudaSuccess;
    prm.m = p.m;
    prm.n = p.n;
    prm.ldc = p.ldc;
    prm.alpha = p.alpha;
    prm.beta = p.beta;
    prm.C = p.C;
    prm.tiles_m = p.tiles_m;
    prm.tiles_n = p.tiles_n;
    prm.total_tiles = p.tiles_m * p.tiles_n;
    prm.ktiles = (int32_t)ceil_div(k, CF::BK);
    prm.a_mn = a_mn;
    prm.b_mn = b_mn;
    prm.err = h->dev_error;
    prm.test_stall = h->test_stall;
    *used = true;
    if constexpr (DEC)
        return launch_tma_dec_variant<CF, EARLY>(prm, grid, h->stream);
    else
        return launch_tma_variant<CF>(prm, grid, h->stream);
}

dgt_status launch_dmma_grouped(dgt_context* h, std::vector<Problem>& probs, const std::vector<KSegment>& segs,
                               int32_t* red_flags, size_t red_count) {
    // drop empty problems, lay out the tile prefix
    std::vector<Problem> live;
    live.reserve(probs.size());
    int64_t tiles = 0;
    bool reduces = false, stack0_seen = false;
    for (auto p : probs) {
        if (p.m <= 0 || p.n <= 0) continue;
        if (p.red_role != 0) {
            if (!red_flags) return fail(h, DGT_ERROR_INVALID_VALUE, "stack reduction without counters");
            // a partial numbered after a stack-0 tile could be waited for by a CTA it needs
            if (p.red_role == 1 && stack0_seen)
                return fail(h, DGT_ERROR_INVALID_VALUE, "partial problem after a stack-0 problem");
            stack0_seen |= p.red_role == 2;
            reduces = true;
        }
        p.tiles_m = (int32_t)ceil_div(p.m, BM);
        p.tiles_n = (int32_t)ceil_div(p.n, BN);
        p.tile_begin = (int32_t)tiles;
        tiles += (int64_t)p.tiles_m * p.tiles_n;
        live.push_back(p);
    }
    if (live.empty()) return DGT_SUCCESS;
    if (tiles > INT32_MAX) return fail(h, DGT_ERROR_INVALID_VALUE, "problem too large (tile count exceeds 2^31)");

    static thread_local GroupedParams prm;  // large; filled per launch (launch copies the value)
    prm.nprob = (int)live.size();
    prm.total_tiles = (int)tiles;
    prm.red_flags = reduces ? red_flags : nullptr;
    prm.err = h->dev_error;
    prm.test_stall = h->test_stall;
    if ((int)live.size() <= MAX_INLINE_PROBS && (int)segs.size() <= MAX_INLINE_SEGS) {
        prm.probs = nullptr;
        prm.segs = nullptr;
        std::copy(live.begin(), live.end(), prm.inl_probs);
        std::copy(segs.begin(), segs.end(), prm.inl_segs);
    } else {
        // device table from the handle's cache: a repeated grouped call (e.g. replayed from a
        // CUDA graph) needs no copy
        const void* parts[2] = {live.data(), segs.data()};
        const size_t bytes[2] = {live.size() * sizeof(Problem), segs.size() * sizeof(KSegment)};
        size_t offs[2];
        void* table = nullptr;
        dgt_status st = device_table(h, 2, parts, bytes, &table, offs);
        if (st != DGT_SUCCESS) return st;
        prm.probs = (const Problem*)((char*)table + offs[0]);
        prm.segs = (const KSegment*)((char*)table + offs[1]);
    }
    int grid = (int)std::min<int64_t>(tiles, h->num_sms);
    cudaError_t e = cudaSuccess;
    if (reduces) DGT_CUDA_TRY(h, cudaMemsetAsync(red_flags, 0, red_count * sizeof(int32_t), h->stream));
    int variant = h->dmma_variant;
    if (variant >= 14 && variant <= 22) {
        bool used = false;
        if (live.size() == 1 && segs.size() == 1 && !reduces) {
            switch (variant) {
                case 14: e = try_tma<T14>(h, live[0], segs[0], grid, &used); break;
                case 15: e = try_tma<T15>(h, live[0], segs[0], grid, &used); break;
                case 16: e = try_tma<T16>(h, live[0], segs[0], grid, &used); break;
                case 17: e = try_tma<T17>(h, live[0], segs[0], grid, &used); break;
                case 18: e = try_tma<T14, true>(h, live[0], segs[0], grid, &used); break;
                case 19: e = try_tma<T17, true>(h, live[0], segs[0], grid, &used); break;
                case 20: e = try_tma<T16, true>(h, live[0], segs[0], grid, &used); break;
                case 21: e = try_tma<T21, true>(h, live[0], segs[0], grid, &used); break;
                default: e = try_tma<T14, true, true>(h, live[0], segs[0], grid, &used); break;
            }
        }
        if (used) {
            h->launches.fetch_add(1);
            if (e != cudaSuccess) return cuda_fail(h, e, "dmma_tma_kernel launch");
            return DGT_SUCCESS;
        }
        variant = variant == 18                                      ? 23
                  : (variant == 14 || variant == 21 || variant == 22) ? 2
                  : variant == 15                                     ? 1
                  : (variant == 16 || variant == 20)                  ? 7
                                                                      : 17;
    }
    switch (variant) {
        case 23: e = launch_variant<V2, true>(prm, grid, h->stream, reduces); break;
        case 24: e = launch_variant<V1, true>(prm, grid, h->stream, reduces); break;
        case 25: e = launch_variant<T17, true>(prm, grid, h->stream, reduces); break;
        case 17: e = launch_variant<T17>(prm, grid, h->stream, reduces); break;
        case 1: e = launch_variant<V1>(prm, grid, h->stream, reduces); break;
        case 2: e = launch_variant<V2>(prm, grid, h->stream, reduces); break;
        case 3: e = launch_variant<V3>(prm, grid, h->stream, reduces); break;
        case 4: e = launch_variant<V4>(prm, grid, h->stream, reduces); break;
        case 5: e = launch_variant<V5>(prm, grid, h->stream, reduces); break;
        case 6: e = launch_variant<V6>(prm, grid, h->stream, reduces); break;
        case 7: e = launch_variant<V7>(prm, grid, h->stream, reduces); break;
        case 8: e = launch_variant<V8>(prm, grid, h->stream, reduces); break;
        case 9: e = launch_variant<V9>(prm, grid, h->stream, reduces); break;
        case 10: e = launch_variant<V10>(prm, grid, h->stream, reduces); break;
        case 11: e = launch_variant<V11>(prm, grid, h->stream, reduces); break;
        case 12: e = launch_variant<V12>(prm, grid, h->stream, reduces); break;
        case 13: e = launch_variant<V13>(prm, grid, h->stream, reduces); break;
        default: e = launch_variant<V0>(prm, grid, h->stream, reduces); break;
    }
    h->launches.fetch_add(1);
    if (e != cudaSuccess) return cuda_fail(h, e, "dmma_grouped_kernel launch");
    return DGT_SUCCESS;
}

}  // namespace dgt
