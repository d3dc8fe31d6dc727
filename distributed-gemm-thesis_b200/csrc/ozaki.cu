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
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include "dgt_internal.cuh"

namespace dgt {
namespace oz {

constexpr int TM = 128, TN = 256, TKB = 128;  // tile rows, tile cols, K bytes per stage
constexpr int STAGES = 4;
constexpr int THREADS = 192;
constexpr int A_STAGE = TM * TKB;  // 16 KB
constexpr int B_STAGE = TN * TKB;  // 32 KB
constexpr uint32_t TMEM_COLS = 512;
constexpr int EXP_NONFINITE = 0x7fff;
constexpr long long WAIT_BUDGET = 4000000000LL;  // clock64 cycles (~2 s) per wait
constexpr int GROUP_M = 8;

struct Seg {
    int32_t a, b;       // digit-plane indices (0-based) of A and B
    int32_t kb0, kb1;   // k-block range [kb0, kb1) in units of TKB bytes
};
struct Group {
    int32_t seg0, seg1;  // segments [seg0, seg1)
    int32_t d;           // diagonal (1-based digit indices s + t)
    int32_t pad;
};

struct Params {
    int64_t m, n, ldc;
    int32_t m_pad, n_pad;
    int32_t tiles_m, tiles_n;
    int32_t ngroups;
    double alpha, beta;
    double* C;
    const int32_t* row_exp;
    const int32_t* col_exp;
    const Seg* segs;
    const Group* groups;
    unsigned int* err;
};

// ---- small PTX wrappers --------------------------------------------------------------------
__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait.  Returns false (and raises the CTA abort flag + device error word) when the
// budget runs out or another role already aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                          unsigned int* err) {
    long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > WAIT_BUDGET) {
            *abort_flag = 1;
            atomicOr(err, DGT_DEVERR_TIMEOUT);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int32_t x, int32_t y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
            "r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// K-major operand tile in shared memory, 128-byte swizzle: rows of 128 bytes, 8-row
// groups 1024 bytes apart (stride byte offset), SM100 descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                  // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset
    d |= (uint64_t)1 << 46;                  // descriptor version (sm100)
    d |= (uint64_t)2 << 61;                  // SWIZZLE_128B
    return d;
}

// Instruction descriptor: kind::i8, D = S32, A = B = signed 8-bit, both K-major, M=128, N=256.
constexpr uint32_t IDESC_I8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                              ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// 2^e for e in [-1022, 1023], built from the exponent field.
__device__ __forceinline__ double pow2i(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// x * 2^e for any e (at most three exact power-of-two steps).
__device__ __forceinline__ double scale2(double x, int e) {
    while (e > 1000) {
        x *= pow2i(1000);
        e -= 1000;
    }
    while (e < -1000) {
        x *= pow2i(-1000);
        e += 1000;
    }
    return x * pow2i(e);
}

// e with max in [2^(e-1), 2^e) from the bit pattern of max = |x|max (0 -> 0, inf/nan -> marker)
__device__ __forceinline__ int exponent_of_max(unsigned long long bits) {
    if (bits == 0ull) return 0;
    if (bits >= 0x7ff0000000000000ull) return EXP_NONFINITE;
    int ef = (int)(bits >> 52);
    if (ef == 0) return (64 - __clzll((long long)bits)) - 1074;  // subnormal
    return ef - 1022;
}

// ---- split kernels ---------------------------------------------------------------------------

// Per-mn max |x| as the bit pattern of |x| (monotone for non-negative doubles).
// MN-contiguous operand: element (mn, kk) at X[mn + kk*ld]; one thread per mn, K split over y.
__global__ void amax_mn_contig(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K, int kchunk,
                               unsigned long long* __restrict__ amax) {
    int64_t mn = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (mn >= MN) return;
    int64_t k0 = (int64_t)blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
    unsigned long long mx = 0;
    for (int64_t kk = k0; kk < k1; ++kk) {
        unsigned long long b = (unsigned long long)__double_as_longlong(X[mn + kk * ld]) & 0x7fffffffffffffffull;
        mx = b > mx ? b : mx;
    }
    if (mx) atomicMax(amax + mn, mx);
}

// K-contiguous operand: element (mn, kk) at X[kk + mn*ld]; one warp per mn.
__global__ void amax_k_contig(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                              unsigned long long* __restrict__ amax) {
    int64_t mn = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
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
    if (lane == 0) amax[mn] = mx;
}

// Digit planes: plane s holds digit s+1 of every element as int8 at [s][mn][kk] (K-major,
// row length k_pad, mn_pad rows); padding rows/columns are written as 0.  Each thread
// produces 32 consecutive kk of one mn.  Thread (mn) also writes exps[mn] once.
template <bool K_CONTIG>
__global__ void __launch_bounds__(128) split_digits(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                                    int64_t mn_pad, int64_t k_pad, int S,
                                                    const unsigned long long* __restrict__ amax,
                                                    int32_t* __restrict__ exps, int8_t* __restrict__ planes) {
    const int64_t mn = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t k0 = (int64_t)blockIdx.y * 32;
    if (mn >= mn_pad) return;
    double v[32];
    int e = 0;
    if (mn < MN) {
        e = exponent_of_max(amax[mn]);
        if (blockIdx.y == 0) exps[mn] = e;
    }
    const bool live = (mn < MN) && (e != EXP_NONFINITE);
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        int64_t kk = k0 + i;
        double x = 0.0;
        if (live && kk < K) x = K_CONTIG ? X[kk + mn * ld] : X[mn + kk * ld];
        v[i] = live ? scale2(x, 7 - e) : 0.0;  // in (-128, 128)
    }
    int8_t* out = planes + mn * k_pad + k0;
    const int64_t plane = mn_pad * k_pad;
    for (int s = 0; s < S; ++s) {
        uint32_t w[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) w[q] = 0;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            int dgt = __double2int_rz(v[i]);          // truncation toward zero: |dgt| <= 127
            v[i] = (v[i] - (double)dgt) * 128.0;     // exact remainder, rescaled
            w[i >> 2] |= ((uint32_t)(uint8_t)(int8_t)dgt) << (8 * (i & 3));
        }
        uint4* o4 = reinterpret_cast<uint4*>(out + s * plane);
        o4[0] = make_uint4(w[0], w[1], w[2], w[3]);
        o4[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

// ---- the INT8 tcgen05 GEMM ---------------------------------------------------------------------

__global__ void __launch_bounds__(THREADS, 1)
    ozaki_i8_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                  const __grid_constant__ Params P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES * A_STAGE;
    uint64_t* bars = (uint64_t*)(sB + STAGES * B_STAGE);
    // bars: full[STAGES], empty[STAGES], acc_full[2], acc_empty[2], done
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 5);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    int32_t* col_exp_all = (int32_t*)(tmem_slot + 4);  // TN entries per epilogue warp

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto full = [&](int s) { return su32(bars + s); };
    auto empty = [&](int s) { return su32(bars + STAGES + s); };
    auto accf = [&](int b) { return su32(bars + 2 * STAGES + b); };
    auto acce = [&](int b) { return su32(bars + 2 * STAGES + 2 + b); };
    const uint32_t done_bar = su32(bars + 2 * STAGES + 4);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(accf(b), 1);
            mbar_init(acce(b), 4);
        }
        mbar_init(done_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(su32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const int total_tiles = P.tiles_m * P.tiles_n;
    auto tile_coords = [&](int tile, int& tm, int& tn) {
        int in_group = GROUP_M * P.tiles_n;
        int grp = tile / in_group;
        int first_m = grp * GROUP_M;
        int gsize = min(P.tiles_m - first_m, GROUP_M);
        tm = first_m + (tile % in_group) % gsize;
        tn = (tile % in_group) / gsize;
    };

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < total_tiles && ok; tile += gridDim.x) {
                int tm, tn;
                tile_coords(tile, tm, tn);
                for (int g = 0; g < P.ngroups && ok; ++g) {
                    const Group G = P.groups[g];
                    for (int si = G.seg0; si < G.seg1 && ok; ++si) {
                        const Seg sg = P.segs[si];
                        for (int kb = sg.kb0; kb < sg.kb1; ++kb) {
                            const int s = it % STAGES;
                            const uint32_t ph = (it / STAGES) & 1;
                            if (!mbar_wait(empty(s), ph ^ 1, abort_flag, P.err)) {
                                ok = false;
                                break;
                            }
                            mbar_expect_tx(full(s), A_STAGE + B_STAGE);
                            tma_load_2d(su32(sA + s * A_STAGE), &tmA, kb * TKB, sg.a * P.m_pad + tm * TM, full(s));
                            tma_load_2d(su32(sB + s * B_STAGE), &tmB, kb * TKB, sg.b * P.n_pad + tn * TN, full(s));
                            ++it;
                        }
                    }
                }
            }
            // drain: wait for this CTA's own loads still in flight (bounded)
            if (!ok) {
                for (uint32_t j = (it > STAGES ? it - STAGES : 0); j < it; ++j) {
                    long long t0 = clock64();
                    while (!mbar_try(full(j % STAGES), (j / STAGES) & 1) && clock64() - t0 < WAIT_BUDGET) {
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            uint32_t it = 0, gcount = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < total_tiles && ok; tile += gridDim.x) {
                for (int g = 0; g < P.ngroups && ok; ++g, ++gcount) {
                    const Group G = P.groups[g];
                    const int b = gcount & 1;
                    const uint32_t u = gcount >> 1;
                    if (!mbar_wait(acce(b), (u & 1) ^ 1, abort_flag, P.err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + (uint32_t)(b * TN);
                    uint32_t acc = 0;
                    for (int si = G.seg0; si < G.seg1 && ok; ++si) {
                        const Seg sg = P.segs[si];
                        for (int kb = sg.kb0; kb < sg.kb1; ++kb) {
                            const int s = it % STAGES;
                            const uint32_t ph = (it / STAGES) & 1;
                            if (!mbar_wait(full(s), ph, abort_flag, P.err)) {
                                ok = false;
                                break;
                            }
                            tc_fence_after();
                            const uint64_t ad = smem_desc_sw128(su32(sA + s * A_STAGE));
                            const uint64_t bd = smem_desc_sw128(su32(sB + s * B_STAGE));
#pragma unroll
                            for (int kk = 0; kk < TKB / 32; ++kk) {
                                // advance 32 bytes (one K=32 step) inside the 128-byte swizzle atom
                                mma_i8(d_tmem, ad + (uint64_t)(kk * 2), bd + (uint64_t)(kk * 2), IDESC_I8, acc);
                                acc = 1;
                            }
                            tc_commit(empty(s));
                            ++it;
                        }
                    }
                    if (ok) tc_commit(accf(b));
                }
            }
            // every MMA this CTA issued has completed once done_bar flips
            tc_commit(done_bar);
            long long t0 = clock64();
            while (!mbar_try(done_bar, 0) && clock64() - t0 < WAIT_BUDGET) {
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: TMEM -> FP64 -> C ----------------
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        const int r_in = q * 32 + lane;
        int32_t* col_exp_s = col_exp_all + (warp - 2) * TN;
        uint32_t gcount = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < total_tiles && ok; tile += gridDim.x) {
            int tm, tn;
            tile_coords(tile, tm, tn);
            const int64_t row = (int64_t)tm * TM + r_in;
            const int64_t n0 = (int64_t)tn * TN;
            // each epilogue warp keeps its own copy of the tile's column exponents, so warps
            // never wait on one another (a warp that aborts cannot strand the others)
            __syncwarp();
            for (int c = lane; c < TN; c += 32) col_exp_s[c] = (n0 + c < P.n) ? P.col_exp[n0 + c] : 0;
            __syncwarp();
            const bool row_ok = row < P.m;
            const int e_row = row_ok ? P.row_exp[row] : 0;
            for (int g = 0; g < P.ngroups; ++g, ++gcount) {
                const int b = gcount & 1;
                const uint32_t u = gcount >> 1;
                if (!mbar_wait(accf(b), u & 1, abort_flag, P.err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int d = P.groups[g].d;
                for (int ch = 0; ch < TN / 32; ++ch) {
                    uint32_t v[32];
                    tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * TN + ch * 32), v);
                    if (!row_ok) continue;
                    double prev[32];
                    double* cbase = P.C + row + (n0 + ch * 32) * P.ldc;
                    const int64_t rem_cols = P.n - (n0 + ch * 32);
                    const int ncols = rem_cols < 32 ? (int)rem_cols : 32;
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        prev[c] = 0.0;
                        if (c < ncols) {
                            if (g > 0)
                                prev[c] = cbase[c * P.ldc];
                            else if (P.beta != 0.0)
                                prev[c] = P.beta * cbase[c * P.ldc];
                        }
                    }
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        if (c < ncols) {
                            const int ec = col_exp_s[ch * 32 + c];
                            double t;
                            if (e_row == EXP_NONFINITE || ec == EXP_NONFINITE)
                                t = __longlong_as_double(0x7ff8000000000000ll);
                            else
                                t = scale2((double)(int32_t)v[c], e_row + ec - 7 * d);
                            cbase[c * P.ldc] = fma(P.alpha, t, prev[c]);
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(acce(b));
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
}

constexpr size_t SMEM_BYTES = 1024 + (size_t)STAGES * (A_STAGE + B_STAGE) + 256 + 4 * TN * 4;

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// 2D map over the stacked digit planes: [S * rows_pad][k_pad] bytes, box = box_rows x 128 B.
bool make_plane_map(CUtensorMap* map, void* base, int64_t rows_total, int64_t k_pad, int box_rows) {
    auto enc = get_encode();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)k_pad, (cuuint64_t)rows_total};
    cuuint64_t strides[1] = {(cuuint64_t)k_pad};
    cuuint32_t box[2] = {(cuuint32_t)TKB, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace oz

// Builds the flush-group schedule: diagonals from least to most significant, each split
// so that pairs * 127^2 * k_pad < 2^31 (exact INT32 accumulation).
static bool ozaki_schedule(int S, int64_t k_pad, std::vector<oz::Seg>& segs, std::vector<oz::Group>& groups) {
    const int64_t kb = k_pad / oz::TKB;
    const int64_t per_pair = 127LL * 127LL * k_pad;
    if (per_pair > (int64_t)INT32_MAX) return false;
    const int max_pairs = (int)std::max<int64_t>(1, (int64_t)INT32_MAX / per_pair);
    for (int d = S + 1; d >= 2; --d) {  // 1-based digit indices s + t = d
        std::vector<std::pair<int, int>> pairs;
        for (int s = 1; s <= S; ++s) {
            int t = d - s;
            if (t >= 1 && t <= S) pairs.emplace_back(s - 1, t - 1);
        }
        for (size_t i = 0; i < pairs.size(); i += max_pairs) {
            oz::Group g{(int32_t)segs.size(), 0, d, 0};
            for (size_t j = i; j < std::min(pairs.size(), i + (size_t)max_pairs); ++j)
                segs.push_back(oz::Seg{pairs[j].first, pairs[j].second, 0, (int32_t)kb});
            g.seg1 = (int32_t)segs.size();
            groups.push_back(g);
        }
    }
    return true;
}

// Scratch layout of one Ozaki call: planes A | planes B | amax A | amax B | exp A | exp B |
// schedule.  Returns false when the shape is outside what the kernels support.
struct OzakiLayout {
    int64_t m_pad, n_pad, k_pad;
    size_t pa, pb, xa, xb, ea, eb, sb, gb, total;
    std::vector<oz::Seg> segs;
    std::vector<oz::Group> groups;
};

static dgt_status ozaki_layout(dgt_context* h, int S, int64_t m, int64_t n, int64_t k, OzakiLayout& L) {
    L.m_pad = ceil_div(m, oz::TM) * oz::TM;
    L.n_pad = ceil_div(n, oz::TN) * oz::TN;
    L.k_pad = ceil_div(k, oz::TKB) * oz::TKB;
    if (!ozaki_schedule(S, L.k_pad, L.segs, L.groups))
        return fail(h, DGT_ERROR_UNSUPPORTED, "K too large for exact INT32 accumulation of one digit product");
    if ((int64_t)S * std::max(L.m_pad, L.n_pad) > INT32_MAX)
        return fail(h, DGT_ERROR_UNSUPPORTED, "matrix too large for 32-bit TMA coordinates");
    auto up = [](size_t x) { return (x + 1023) / 1024 * 1024; };
    L.pa = up((size_t)S * L.m_pad * L.k_pad);
    L.pb = up((size_t)S * L.n_pad * L.k_pad);
    L.xa = up(m * 8);
    L.xb = up(n * 8);
    L.ea = up(m * 4);
    L.eb = up(n * 4);
    L.sb = up(L.segs.size() * sizeof(oz::Seg));
    L.gb = up(L.groups.size() * sizeof(oz::Group));
    L.total = L.pa + L.pb + L.xa + L.xb + L.ea + L.eb + L.sb + L.gb;
    return DGT_SUCCESS;
}

size_t ozaki_scratch_bytes(int S, int64_t m, int64_t n, int64_t k) {
    OzakiLayout L;
    return ozaki_layout(nullptr, S, m, n, k, L) == DGT_SUCCESS ? L.total : 0;
}

// The Ozaki INT8 path on caller-provided scratch (L.total bytes at ws).  h may be null:
// then no profiling marks, launch counts or error messages are recorded.
static dgt_status ozaki_run(dgt_context* h, cudaStream_t s, int num_sms, unsigned int* err, void* ws,
                            const OzakiLayout& L, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                            const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                            int64_t ldc, int S) {
    const int64_t m_pad = L.m_pad, n_pad = L.n_pad, k_pad = L.k_pad;
    char* p = (char*)ws;
    int8_t* planesA = (int8_t*)p;
    int8_t* planesB = (int8_t*)(p + L.pa);
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

    DGT_CUDA_TRY(h, cudaMemcpyAsync(dsegs, L.segs.data(), L.segs.size() * sizeof(oz::Seg), cudaMemcpyHostToDevice,
                                    s));
    DGT_CUDA_TRY(h, cudaMemcpyAsync(dgroups, L.groups.data(), L.groups.size() * sizeof(oz::Group),
                                    cudaMemcpyHostToDevice, s));
    if (h) mark(h, 0);
    DGT_CUDA_TRY(h, cudaMemsetAsync(amaxA, 0, m * 8, s));
    DGT_CUDA_TRY(h, cudaMemsetAsync(amaxB, 0, n * 8, s));

    // op(A) is m x k: 'N' -> element (i,kk) at A[i + kk*lda] (MN-contiguous); 'T' -> A[kk + i*lda]
    // op(B) as its transpose n x k: 'N' -> element (j,kk) at B[kk + j*ldb] (K-contiguous); 'T' -> B[j + kk*ldb]
    auto amax = [&](const double* X, int64_t ld, int64_t MN, bool kcontig, unsigned long long* out) {
        if (kcontig) {
            oz::amax_k_contig<<<(unsigned)ceil_div(MN, 8), 256, 0, s>>>(X, ld, MN, k, out);
        } else {
            int kchunk = 512;
            dim3 grid((unsigned)ceil_div(MN, 256), (unsigned)ceil_div(k, kchunk));
            oz::amax_mn_contig<<<grid, 256, 0, s>>>(X, ld, MN, k, kchunk, out);
        }
        return counted("ozaki amax");
    };
    auto split = [&](const double* X, int64_t ld, int64_t MN, int64_t mn_pad, bool kcontig,
                     const unsigned long long* am, int32_t* ex, int8_t* planes) {
        dim3 grid((unsigned)ceil_div(mn_pad, 128), (unsigned)(k_pad / 32));
        if (kcontig)
            oz::split_digits<true><<<grid, 128, 0, s>>>(X, ld, MN, k, mn_pad, k_pad, S, am, ex, planes);
        else
            oz::split_digits<false><<<grid, 128, 0, s>>>(X, ld, MN, k, mn_pad, k_pad, S, am, ex, planes);
        return counted("ozaki split");
    };
    dgt_status st;
    if ((st = amax(A, lda, m, ta, amaxA)) != DGT_SUCCESS) return st;
    if ((st = amax(B, ldb, n, !tb, amaxB)) != DGT_SUCCESS) return st;
    if ((st = split(A, lda, m, m_pad, ta, amaxA, expA, planesA)) != DGT_SUCCESS) return st;
    if ((st = split(B, ldb, n, n_pad, !tb, amaxB, expB, planesB)) != DGT_SUCCESS) return st;

    CUtensorMap tmA, tmB;
    if (!oz::make_plane_map(&tmA, planesA, (int64_t)S * m_pad, k_pad, oz::TM) ||
        !oz::make_plane_map(&tmB, planesB, (int64_t)S * n_pad, k_pad, oz::TN))
        return fail(h, DGT_ERROR_CUDA, "cuTensorMapEncodeTiled failed");

    static bool attr = false;
    if (!attr) {
        DGT_CUDA_TRY(h, cudaFuncSetAttribute(oz::ozaki_i8_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)oz::SMEM_BYTES));
        attr = true;
    }
    oz::Params prm{};
    prm.m = m;
    prm.n = n;
    prm.ldc = ldc;
    prm.m_pad = (int32_t)m_pad;
    prm.n_pad = (int32_t)n_pad;
    prm.tiles_m = (int32_t)(m_pad / oz::TM);
    prm.tiles_n = (int32_t)(n_pad / oz::TN);
    prm.ngroups = (int32_t)L.groups.size();
    prm.alpha = alpha;
    prm.beta = beta;
    prm.C = C;
    prm.row_exp = expA;
    prm.col_exp = expB;
    prm.segs = dsegs;
    prm.groups = dgroups;
    prm.err = err;
    const int tiles = prm.tiles_m * prm.tiles_n;
    const int grid = std::min(tiles, num_sms);
    if (h) mark(h, 1);
    oz::ozaki_i8_gemm<<<grid, oz::THREADS, oz::SMEM_BYTES, s>>>(tmA, tmB, prm);
    if ((st = counted("ozaki_i8_gemm")) != DGT_SUCCESS) return st;
    if (h) mark(h, 2);
    return DGT_SUCCESS;
}

dgt_status ozaki_dgemm_on(cudaStream_t s, int num_sms, unsigned int* err, void* ws, size_t ws_bytes, bool ta,
                          bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                          const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int S) {
    OzakiLayout L;
    dgt_status st = ozaki_layout(nullptr, S, m, n, k, L);
    if (st != DGT_SUCCESS) return st;
    if (L.total > ws_bytes) return DGT_ERROR_INVALID_VALUE;
    return ozaki_run(nullptr, s, num_sms, err, ws, L, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, S);
}

dgt_status ozaki_dgemm(dgt_context* h, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                       const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                       int64_t ldc, dgt_fp64_mode mode, int S) {
    if (mode != DGT_FP64_OZAKI_INT8)
        return fail(h, DGT_ERROR_UNSUPPORTED, "this build implements the INT8 Ozaki path only");
    OzakiLayout L;
    dgt_status st = ozaki_layout(h, S, m, n, k, L);
    if (st != DGT_SUCCESS) return st;
    void* ws = nullptr;
    st = ensure_workspace(h, L.total, &ws, 0);
    if (st != DGT_SUCCESS) return st;
    return ozaki_run(h, h->stream, h->num_sms, h->dev_error, ws, L, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C,
                     ldc, S);
}

}  // namespace dgt

extern "C" dgt_status dgt_sgemm(dgt_handle_t h, char, char, int64_t, int64_t, int64_t, const float*, const float*,
                                int64_t, const float*, int64_t, const float*, float*, int64_t, dgt_fp32_mode) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    return dgt::fail(h, DGT_ERROR_UNSUPPORTED, "sgemm is not built yet");
}
