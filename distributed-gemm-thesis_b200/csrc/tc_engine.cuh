// The tcgen05 "digit GEMM" engine shared by the FP64 emulation (ozaki.cu) and the FP32
// split GEMMs (sgemm.cu): C (+)= sum over flush groups of sums of digit-plane products,
// operands staged by TMA from K-major planes, products in TMEM, folded by an epilogue.
//
// Persistent, one 128 x 256 output tile per CTA at a time, warp-specialised: warp 0 issues
// TMA loads of the planes (swizzled boxes, STAGES-deep mbarrier ring), warp 1 issues
// tcgen05.mma (M=128, N=256, K=32 bytes per instruction) into one of two 256-column TMEM
// accumulators, the epilogue warps drain the other accumulator (tcgen05.ld.32x32b.x32) into
// C while the next group multiplies.  Every mbarrier wait has an iteration budget; on
// expiry the kernel records DGT_DEVERR_TIMEOUT, stops all roles, waits for its own MMAs and
// loads, frees TMEM and returns.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "dgt_internal.cuh"

namespace dgt {
namespace oz {

constexpr int TM = 128, TN = 256;  // output tile
constexpr int KPAD = 128;          // K of the digit planes is padded to a multiple of this
constexpr uint32_t TMEM_COLS = 512;

// Kernel variants (the autotuner's knob): epilogue warps (4 or 8), K bytes per pipeline
// stage (128 with 128-byte swizzle, or 64 with 64-byte swizzle), ring depth.
// PAIR: a cluster of two CTAs shares one M=256 x N=256 tcgen05.mma (cta_group::2); each CTA
// stages its 128 rows of A and half (128 rows) of B, so per-SM B traffic halves.
template <int EPI_, int TKB_, int STAGES_, bool PAIR_ = false>
struct OzCfg {
    static constexpr int EPI = EPI_, TKB = TKB_, STAGES = STAGES_;
    static constexpr bool PAIR = PAIR_;
    static constexpr int THREADS = 64 + 32 * EPI;
    static constexpr int A_STAGE = TM * TKB, B_STAGE = (PAIR ? TN / 2 : TN) * TKB;
    static constexpr int TILE_M = PAIR ? 2 * TM : TM;  // rows of output per (cluster) tile
    static constexpr size_t SMEM = 1024 + (size_t)STAGES * (A_STAGE + B_STAGE) + 256 + (size_t)EPI * TN * 4 + 512;
};
constexpr int UNIT_RING = 8;  // depth of the dynamic scheduler's unit ring (see digit_gemm)
constexpr int EXP_NONFINITE = 0x7fff;
constexpr long long WAIT_BUDGET = 4000000000LL;  // clock64 cycles (~2 s) per wait
constexpr int GROUP_M = 8;

struct Seg {
    int32_t a, b;       // digit-plane indices (0-based) of A and B
    int32_t kb0, kb1;   // k-block range [kb0, kb1) in units of the kernel's stage depth
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
    const Seg* segs_ext;      // schedule in device memory when it exceeds the inline tables
    const Group* groups_ext;
    unsigned int* err;
    float* Cf;  // FP32 output (EPI_MODE 1)
    float alpha_f, beta_f;
    // EPI_MODE 2: group g's accumulator reduced modulo its modulus (Group::pad) is stored as
    // one byte per element at res[g * res_plane + row + col * res_ld]
    uint8_t* res;
    int64_t res_ld, res_plane;
    // The schedule travels inside the launch's parameters (so a captured CUDA graph needs
    // no host-to-device copy); MAX_SEGS / MAX_GROUPS keep the block under 32 KB.
    Seg segs[640];
    Group groups[640];
    // grouped mode: per-problem descriptors in device memory, tiles numbered problem by problem;
    // prob_tiles[p] = gprobs[p].tile_begin as a compact array (the binary search per work unit
    // stays in one or two cache lines)
    const struct GProb* gprobs;
    const int32_t* prob_tiles;
    int32_t nprob, total_tiles;
    // Failure-path test hook (DGT_TUNE_TEST_STALL): nonzero makes every CTA's producer
    // withhold the operand loads of its first pipeline stage, a barrier phase nothing
    // completes, so the MMA issuer's first wait runs out of its budget.  No load or MMA is in
    // flight for that stage, so the abort path drains and returns as on a real stall.
    int32_t test_stall;
    // Dynamic unit order: when set, the clusters take work units from this zeroed counter
    // (atomicAdd) in ascending order instead of a static round robin.
    int32_t* sched;
};
constexpr int MAX_SEGS = 640, MAX_GROUPS = 640;

// One problem of a grouped launch: its planes' tensor maps, pads, output and scales.  A
// segment whose kb1 is negative runs to the problem's own end of K (nkb stages).
struct alignas(64) GProb {
    CUtensorMap tmA, tmB;
    int64_t m, n, ldc;
    double* C;
    const int32_t* row_exp;
    const int32_t* col_exp;
    double alpha, beta;
    int32_t m_pad, n_pad, nkb, tiles_m, tiles_n, tile_begin;
    uint8_t* res;  // EPI_MODE 2: residue planes of this product
    int64_t res_ld, res_plane;
};

// The tile a role works on: its coordinates and, in grouped mode, its problem descriptor
// (fields are read through the kernel's accessors, so nothing is copied into registers).
struct TileCtx {
    const GProb* gp;
    int32_t tm, tn;
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
// try_wait with a suspend-time hint: a waiting warp sleeps until the phase completes (or
// ~1 ms passes) instead of spinning.  Spinning epilogue warps (eight per SM while the MMAs
// run) drew power under the cap: with the hint a 16384^3 CRT product runs 2.8 % faster
// (68.5 vs 70.5 ms, same box, alternating runs).  Waits stay bounded by the caller's budget.
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(1000000u)
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

// Cluster-scope forms for barriers that the other CTA of a pair may arrive on.
__device__ __forceinline__ bool mbar_try_cluster(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(1000000u)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                                  unsigned int* err) {
    long long t0 = clock64();
    while (!mbar_try_cluster(bar, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > WAIT_BUDGET) {
            *abort_flag = 1;
            atomicOr(err, DGT_DEVERR_TIMEOUT);
            return false;
        }
    }
    return true;
}
// Arrive (release, cluster scope) on a barrier given by its shared::cluster address.
__device__ __forceinline__ void mbar_arrive_release_cluster(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ void st_cluster_s32(uint32_t cluster_addr, int32_t v) {
    asm volatile("st.shared::cluster.s32 [%0], %1;\n" ::"r"(cluster_addr), "r"(v) : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int32_t x, int32_t y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
            "r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, int32_t x, int32_t y,
                                                 uint32_t leader_bar) {
    // both CTAs of the pair load into their own shared memory; bytes complete on the
    // leader's barrier (no multicast)
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
        "%3}], [%4];\n" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(leader_bar)
        : "memory");
}

__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;\n" ::"l"(map) : "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
    return r;
}

// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t map_to_rank(uint32_t addr, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(out) : "r"(addr), "r"(rank));
    return out;
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];\n" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Commit of the pair's MMAs, arriving on the barrier at the same offset in every CTA of mask.
__device__ __forceinline__ void tc_commit_pair(uint32_t bar, uint16_t mask) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;\n" ::"r"(
                     bar),
                 "h"(mask)
                 : "memory");
}

__device__ __forceinline__ void mma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_bf16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                              uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
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

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// K-major operand tile in shared memory with the swizzle the TMA box used: rows of TKB
// bytes (128 -> SWIZZLE_128B, 64 -> SWIZZLE_64B), 8-row groups 8*TKB bytes apart (stride
// byte offset), SM100 descriptor version 1.
template <int TKB>
__device__ __forceinline__ uint64_t smem_desc_k(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                        // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)((8 * TKB) >> 4) << 32;         // stride byte offset
    d |= (uint64_t)1 << 46;                        // descriptor version (sm100)
    d |= (uint64_t)(TKB == 128 ? 2 : 4) << 61;     // SWIZZLE_128B or SWIZZLE_64B
    return d;
}

// Instruction descriptor: kind::i8, D = S32, A = B = signed 8-bit, both K-major, M=128, N=256.
constexpr uint32_t IDESC_I8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                              ((uint32_t)(TM >> 4) << 24);

// The pair's M=256 forms of both descriptors.
constexpr uint32_t IDESC_I8_PAIR = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                                   ((uint32_t)((2 * TM) >> 4) << 24);
constexpr uint32_t IDESC_BF16_PAIR = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                                     ((uint32_t)((2 * TM) >> 4) << 24);

// Instruction descriptor: kind::f16, D = F32, A = B = BF16, both K-major, M=128, N=256.
constexpr uint32_t IDESC_BF16 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
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

// 64 consecutive 32-bit columns of this warp's 32 TMEM lanes, load and wait in one asm (the
// registers are written asynchronously until the wait, so nothing may touch them in between).
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t (&v)[64]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
        : "r"(taddr)
        : "memory");
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

// KIND: 0 = INT8 digits (kind::i8, INT32 accumulator), 1 = BF16 operands (kind::f16, FP32
// accumulator).  EPI: 0 = FP64 fold C = beta*C + alpha*sum_g 2^(e_i+f_j-7d_g) P_g,
// 1 = FP32 output C = alpha*acc + beta*C (a single flush group), 2 = residues: each group's
// INT32 accumulator modulo the group's modulus, one byte per element (CRT emulation).
template <class CF, int KIND, int EPI_MODE, bool GROUPED = false>
__global__ void __launch_bounds__(CF::THREADS, 1)
    digit_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               const __grid_constant__ Params P) {
    constexpr int STAGES = CF::STAGES, TKB = CF::TKB, A_STAGE = CF::A_STAGE, B_STAGE = CF::B_STAGE;
    constexpr int EPI = CF::EPI;
    constexpr bool PAIR = CF::PAIR;
    constexpr int TILE_M = CF::TILE_M;
    const uint32_t crank = PAIR ? cluster_rank() : 0;  // 0 = leader (issues the MMAs)
    const bool leader = crank == 0;
    const int unit = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;  // cluster (or CTA) index
    const int units = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;
    const Seg* SEGS = P.segs_ext ? P.segs_ext : P.segs;
    const Group* GROUPS = P.groups_ext ? P.groups_ext : P.groups;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES * A_STAGE;
    uint64_t* bars = (uint64_t*)(sB + STAGES * B_STAGE);
    // bars: full[STAGES], empty[STAGES], acc_full[2], acc_empty[2], done
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 5);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    int32_t* col_exp_all = (int32_t*)(tmem_slot + 4);  // TN entries per epilogue warp
    // dynamic unit order (P.sched): the leader's producer takes units from the global counter
    // and publishes them through this ring to every role of both CTAs of the cluster
    volatile int32_t* uring = col_exp_all + EPI * TN;            // UNIT_RING unit ids
    uint64_t* ubars = (uint64_t*)(col_exp_all + EPI * TN + UNIT_RING);  // ufull[R], uempty[R]
    // grouped mode: problems whose tensor maps this CTA's producer has already acquired
    constexpr int ACQ_BITS = 2048;
    uint32_t* acquired = (uint32_t*)(ubars + 2 * UNIT_RING);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto full = [&](int s) { return su32(bars + s); };
    auto empty = [&](int s) { return su32(bars + STAGES + s); };
    auto accf = [&](int b) { return su32(bars + 2 * STAGES + b); };
    auto acce = [&](int b) { return su32(bars + 2 * STAGES + 2 + b); };
    const uint32_t done_bar = su32(bars + 2 * STAGES + 4);
    auto ufull = [&](int r) { return su32(ubars + r); };
    auto uempty = [&](int r) { return su32(ubars + UNIT_RING + r); };
    const bool dyn = P.sched != nullptr;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(accf(b), 1);
            mbar_init(acce(b), PAIR ? 2 * EPI : EPI);  // the leader's counts both CTAs' epilogue warps
        }
        mbar_init(done_bar, 1);
        for (int r = 0; r < UNIT_RING; ++r) {
            mbar_init(ufull(r), 1);
            // readers of a slot: the leader's MMA issuer and epilogue warps, and in a pair the
            // other CTA's producer and epilogue warps (the leader's producer writes it)
            mbar_init(uempty(r), PAIR ? 2 + 2 * EPI : 1 + EPI);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 1) {
        if constexpr (PAIR) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                             su32(tmem_slot)),
                         "r"(TMEM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                             su32(tmem_slot)),
                         "r"(TMEM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
        }
    }
    tc_fence_before();
    __syncthreads();
    if constexpr (PAIR) cluster_sync();  // both CTAs' barriers and TMEM exist before any cross-CTA traffic
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const int total_tiles = GROUPED ? P.total_tiles : P.tiles_m * P.tiles_n;
    // Work units.  The residue epilogue (EPI_MODE 2) stores every group -- one CRT modulus --
    // to its own plane, so a unit is one (tile, group) pair, groups outermost: the CTAs then
    // run one modulus at a time over the whole output and share its planes' panels in L2,
    // and the tail after the last full wave is at most one modulus of one tile.  The other
    // modes fold a tile's groups into C in order, so a unit is a whole tile.
    constexpr bool UNIT_PER_GROUP = EPI_MODE == 2;
    const int total_units = UNIT_PER_GROUP ? total_tiles * P.ngroups : total_tiles;
    auto unit_of = [&](int u, int& tile, int& g0, int& g1) {
        if constexpr (UNIT_PER_GROUP) {
            g0 = u / total_tiles;
            tile = u - g0 * total_tiles;
            g1 = g0 + 1;
        } else {
            tile = u;
            g0 = 0;
            g1 = P.ngroups;
        }
    };
    // The j-th unit this CTA (or cluster) works on, or -1 past the last.  Static order: a
    // round robin.  Dynamic order: read from ring slot j once the scheduler has filled it; the
    // slot is then released to the scheduler at once (the id is in a register).
    auto unit_static = [&](uint32_t j) -> int {
        const int un = unit + (int)j * units;
        return un < total_units ? un : -1;
    };
    auto unit_take = [&](uint32_t j, bool& ok) -> int {  // one thread
        const int r = (int)(j % UNIT_RING);
        if (!mbar_wait_cluster(ufull(r), (j / UNIT_RING) & 1, abort_flag, P.err)) {
            ok = false;
            return -1;
        }
        const int un = uring[r];
        mbar_arrive_release_cluster(PAIR ? map_to_rank(uempty(r), 0) : uempty(r));
        return un;
    };
    auto unit_take_warp = [&](uint32_t j, bool& ok) -> int {  // a whole warp: lane 0 takes it
        int un = -1, got = 1;
        if ((threadIdx.x & 31) == 0) {
            bool lok = true;
            un = unit_take(j, lok);
            got = lok;
        }
        un = __shfl_sync(0xffffffffu, un, 0);
        if (!__shfl_sync(0xffffffffu, got, 0)) ok = false;
        return un;
    };
    // The scheduler (the leader's producer lane): the next unit from the counter, published to
    // both CTAs' rings; -1 once the units are exhausted.
    auto unit_publish = [&](uint32_t j, bool& ok) -> int {
        const int r = (int)(j % UNIT_RING);
        if (!mbar_wait_cluster(uempty(r), ((j / UNIT_RING) & 1) ^ 1, abort_flag, P.err)) {
            ok = false;
            return -1;
        }
        int un = atomicAdd(P.sched, 1);
        if (un >= total_units) un = -1;
        uring[r] = un;
        mbar_arrive_release_cluster(ufull(r));
        if constexpr (PAIR) {
            st_cluster_s32(map_to_rank(su32((const void*)(uring + r)), 1), un);
            mbar_arrive_release_cluster(map_to_rank(ufull(r), 1));
        }
        return un;
    };
    auto raster = [](int tile, int tiles_m, int tiles_n) -> int2 {
        int in_group = GROUP_M * tiles_n;
        int grp = tile / in_group;
        int first_m = grp * GROUP_M;
        int gsize = min(tiles_m - first_m, GROUP_M);
        return make_int2(first_m + (tile % in_group) % gsize, (tile % in_group) / gsize);
    };
    auto ctx_of = [&](int tile) -> TileCtx {
        TileCtx c;
        if constexpr (GROUPED) {
            int lo = 0, hi = P.nprob - 1;  // last problem whose first tile is <= tile
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if ((P.prob_tiles ? P.prob_tiles[mid] : P.gprobs[mid].tile_begin) <= tile)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            c.gp = P.gprobs + lo;
            const int2 t = raster(tile - c.gp->tile_begin, c.gp->tiles_m, c.gp->tiles_n);
            c.tm = t.x;
            c.tn = t.y;
        } else {
            c.gp = nullptr;
            const int2 t = raster(tile, P.tiles_m, P.tiles_n);
            c.tm = t.x;
            c.tn = t.y;
        }
        return c;
    };
#define DGT_TILE_FIELD(cx, grouped_expr, single_expr) (GROUPED ? (cx).gp->grouped_expr : P.single_expr)
    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            if constexpr (GROUPED)
                for (int w = 0; w < ACQ_BITS / 32; ++w) acquired[w] = 0u;
            for (uint32_t j = 0; ok; ++j) {
                const int un = !dyn ? unit_static(j) : leader ? unit_publish(j, ok) : unit_take(j, ok);
                if (un < 0) break;
                int tile, g0, g1;
                unit_of(un, tile, g0, g1);
                const TileCtx cx = ctx_of(tile);
                const int tm = cx.tm, tn = cx.tn;
                const CUtensorMap* tA = GROUPED ? &cx.gp->tmA : &tmA;
                const CUtensorMap* tB = GROUPED ? &cx.gp->tmB : &tmB;
                if constexpr (GROUPED) {
                    // the problem's maps reached global memory by a host copy: order them for
                    // the tensor-map proxy before the TMA unit reads them, once per problem
                    const int pi = (int)(cx.gp - P.gprobs);
                    const uint32_t bit = 1u << (pi & 31);
                    if (pi >= ACQ_BITS || !(acquired[pi >> 5] & bit)) {
                        tensormap_acquire(tA);
                        tensormap_acquire(tB);
                        if (pi < ACQ_BITS) acquired[pi >> 5] |= bit;
                    }
                }
                const int m_pad = DGT_TILE_FIELD(cx, m_pad, m_pad), n_pad = DGT_TILE_FIELD(cx, n_pad, n_pad);
                for (int g = g0; g < g1 && ok; ++g) {
                    const Group G = GROUPS[g];
                    for (int si = G.seg0; si < G.seg1 && ok; ++si) {
                        const Seg sg = SEGS[si];
                        const int kb1 = sg.kb1 < 0 ? DGT_TILE_FIELD(cx, nkb, ngroups) : sg.kb1;
                        for (int kb = sg.kb0; kb < kb1; ++kb) {
                            const int s = it % STAGES;
                            const uint32_t ph = (it / STAGES) & 1;
                            if (!mbar_wait(empty(s), ph ^ 1, abort_flag, P.err)) {
                                ok = false;
                                break;
                            }
                            if (P.test_stall && it == 0) {  // withheld: stage 0 never fills
                                ++it;
                                continue;
                            }
                            if constexpr (PAIR) {
                                const uint32_t lbar = map_to_rank(full(s), 0);
                                if (leader) mbar_expect_tx(full(s), 2 * (A_STAGE + B_STAGE));
                                tma_load_2d_pair(su32(sA + s * A_STAGE), tA, kb * TKB,
                                                 sg.a * m_pad + tm * TILE_M + (int)crank * TM, lbar);
                                tma_load_2d_pair(su32(sB + s * B_STAGE), tB, kb * TKB,
                                                 sg.b * n_pad + tn * TN + (int)crank * (TN / 2), lbar);
                            } else {
                                mbar_expect_tx(full(s), A_STAGE + B_STAGE);
                                tma_load_2d(su32(sA + s * A_STAGE), tA, kb * TKB, sg.a * m_pad + tm * TM, full(s));
                                tma_load_2d(su32(sB + s * B_STAGE), tB, kb * TKB, sg.b * n_pad + tn * TN, full(s));
                            }
                            ++it;
                        }
                    }
                }
            }
            // drain: wait for this CTA's own loads still in flight (bounded)
            if (!ok && leader) {
                for (uint32_t j = (it > STAGES ? it - STAGES : 0); j < it; ++j) {
                    if (P.test_stall && j == 0) continue;  // the withheld stage has nothing in flight
                    long long t0 = clock64();
                    while (!mbar_try(full(j % STAGES), (j / STAGES) & 1) && clock64() - t0 < WAIT_BUDGET) {
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (the pair's leader only) ----------------
        if (lane == 0 && leader) {
            uint32_t it = 0, gcount = 0;
            bool ok = true;
            for (uint32_t j = 0; ok; ++j) {
                const int un = dyn ? unit_take(j, ok) : unit_static(j);
                if (un < 0) break;
                int tile, g0, g1;
                unit_of(un, tile, g0, g1);
                const TileCtx cx = ctx_of(tile);
                for (int g = g0; g < g1 && ok; ++g, ++gcount) {
                    const Group G = GROUPS[g];
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
                        const Seg sg = SEGS[si];
                        const int kb1 = sg.kb1 < 0 ? DGT_TILE_FIELD(cx, nkb, ngroups) : sg.kb1;
                        for (int kb = sg.kb0; kb < kb1; ++kb) {
                            const int s = it % STAGES;
                            const uint32_t ph = (it / STAGES) & 1;
                            if (!mbar_wait(full(s), ph, abort_flag, P.err)) {
                                ok = false;
                                break;
                            }
                            tc_fence_after();
                            const uint64_t ad = smem_desc_k<TKB>(su32(sA + s * A_STAGE));
                            const uint64_t bd = smem_desc_k<TKB>(su32(sB + s * B_STAGE));
#pragma unroll
                            for (int kk = 0; kk < TKB / 32; ++kk) {
                                // advance 32 bytes (one K=32 step) inside the swizzle atom
                                const uint64_t a_k = ad + (uint64_t)(kk * 2), b_k = bd + (uint64_t)(kk * 2);
                                if constexpr (PAIR) {
                                    if constexpr (KIND == 0)
                                        mma_i8_pair(d_tmem, a_k, b_k, IDESC_I8_PAIR, acc);
                                    else
                                        mma_bf16_pair(d_tmem, a_k, b_k, IDESC_BF16_PAIR, acc);
                                } else {
                                    if constexpr (KIND == 0)
                                        mma_i8(d_tmem, a_k, b_k, IDESC_I8, acc);
                                    else
                                        mma_bf16(d_tmem, a_k, b_k, IDESC_BF16, acc);
                                }
                                acc = 1;
                            }
                            if constexpr (PAIR)
                                tc_commit_pair(empty(s), 0x3);  // frees the stage in both CTAs
                            else
                                tc_commit(empty(s));
                            ++it;
                        }
                    }
                    if (ok) {
                        if constexpr (PAIR)
                            tc_commit_pair(accf(b), 0x3);  // both CTAs' epilogues may read their rows
                        else
                            tc_commit(accf(b));
                    }
                }
            }
            // every MMA this CTA issued has completed once done_bar flips
            if constexpr (PAIR)
                tc_commit_pair(done_bar, 0x1);
            else
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
        // EPI_MODE 2: lane g keeps group g's modulus constants (read with a shuffle), so the
        // per-group work has no integer division
        uint32_t k_off = 0, k_c16 = 0, k_mg = 0;
        if constexpr (EPI_MODE == 2) {
            if (lane < P.ngroups) {
                const uint32_t pm = (uint32_t)GROUPS[lane].pad;
                k_off = pm * (0x80000000u / pm);
                k_c16 = (1u << 16) % pm;
                k_mg = (uint32_t)(0x100000000ull / pm) + 1u;
            }
        }
        for (uint32_t j = 0; ok; ++j) {
            const int un = dyn ? unit_take_warp(j, ok) : unit_static(j);
            if (un < 0) break;
            int tile, g0, g1;
            unit_of(un, tile, g0, g1);
            const TileCtx cx = ctx_of(tile);
            const int tm = cx.tm, tn = cx.tn;
            const int64_t row = (int64_t)tm * TILE_M + (int64_t)crank * TM + r_in;
            const int64_t n0 = (int64_t)tn * TN;
            // each epilogue warp keeps its own copy of the tile's column exponents, so warps
            // never wait on one another (a warp that aborts cannot strand the others)
            __syncwarp();
            if constexpr (EPI_MODE == 0)
                for (int c = lane; c < TN; c += 32)
                    col_exp_s[c] = (n0 + c < DGT_TILE_FIELD(cx, n, n)) ? DGT_TILE_FIELD(cx, col_exp, col_exp)[n0 + c] : 0;
            __syncwarp();
            const bool row_ok = row < DGT_TILE_FIELD(cx, m, m);
            const int e_row = (EPI_MODE == 0 && row_ok) ? DGT_TILE_FIELD(cx, row_exp, row_exp)[row] : 0;
            for (int g = g0; g < g1; ++g, ++gcount) {
                const int b = gcount & 1;
                const uint32_t u = gcount >> 1;
                if (!mbar_wait(accf(b), u & 1, abort_flag, P.err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int d = GROUPS[g].d;
                // with 8 epilogue warps, two warps share a lane quarter and split the columns
                constexpr int CHUNKS = TN / 32 / (EPI / 4);
                const int ch0 = ((warp - 2) / 4) * CHUNKS;
                if constexpr (EPI_MODE == 2) {
                    // acc mod p in integers.  |acc| <= k_pad 2^14 <= 2^31 - 2^21 (k_pad < 2^17),
                    // so x = acc + off (off = p floor(2^31 / p) >= 2^31 - 256, a multiple of p)
                    // lies in (0, 2^32); t = (x >> 16)(2^16 mod p) + (x & 0xffff) < 2^24 is
                    // congruent to acc, and t / p = umulhi(t, floor(2^32 / p) + 1) exactly for
                    // t < 2^24 (Granlund & Montgomery 1994, thm 4.2)
                    const uint32_t pm = (uint32_t)GROUPS[g].pad;
                    uint32_t off, c16, mg;
                    if (g < 32) {
                        off = __shfl_sync(0xffffffffu, k_off, g);
                        c16 = __shfl_sync(0xffffffffu, k_c16, g);
                        mg = __shfl_sync(0xffffffffu, k_mg, g);
                    } else {
                        off = pm * (0x80000000u / pm);
                        c16 = (1u << 16) % pm;
                        mg = (uint32_t)(0x100000000ull / pm) + 1u;
                    }
                    // Each lane holds one row; the plane is column-major with rows contiguous.
                    // Four columns' bytes of this lane's row form one word; a 4 x 4 byte
                    // transpose across the quad of lanes 4a .. 4a+3 (two shuffle steps) leaves
                    // lane 4a+b with column 4i+b's bytes of rows 4a .. 4a+3, so a warp stores
                    // four columns x 32 rows with one word per lane.  Every lane stores, rows
                    // past m and columns past n included: the plane has m_pad rows and n_pad
                    // columns.
                    const int bq = lane & 3;
                    const uint32_t selA = (bq & 2) ? 0x3276u : 0x5410u;  // swap 16-bit halves with lane ^ 2
                    const uint32_t selB = (bq & 1) ? 0x3715u : 0x6240u;  // swap bytes with lane ^ 1
                    const int64_t rld = DGT_TILE_FIELD(cx, res_ld, res_ld);
                    uint8_t* rbase = DGT_TILE_FIELD(cx, res, res) + (int64_t)g * DGT_TILE_FIELD(cx, res_plane, res_plane) +
                                     (row - lane + 4 * (lane >> 2)) + (n0 + ch0 * 32 + bq) * rld;
                    static_assert(CHUNKS % 2 == 0, "residue epilogue: 64-column TMEM loads");
                    for (int c2 = 0; c2 < CHUNKS / 2; ++c2) {
                        uint32_t v[64];
                        tmem_ld64(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * TN + (ch0 + 2 * c2) * 32), v);
#pragma unroll
                        for (int i = 0; i < 16; ++i) {
                            uint32_t r[4];
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const uint32_t x = v[4 * i + u] + off;
                                const uint32_t t = (x >> 16) * c16 + (x & 0xffffu);
                                r[u] = t - pm * __umulhi(t, mg);
                            }
                            uint32_t wd = __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
                            wd = __byte_perm(wd, __shfl_xor_sync(0xffffffffu, wd, 2), selA);
                            wd = __byte_perm(wd, __shfl_xor_sync(0xffffffffu, wd, 1), selB);
                            *reinterpret_cast<uint32_t*>(rbase + (int64_t)(64 * c2 + 4 * i) * rld) = wd;
                        }
                    }
                }
                for (int ch = ch0; ch < ch0 + CHUNKS && EPI_MODE != 2; ++ch) {
                    uint32_t v[32];
                    tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * TN + ch * 32), v);
                    if (!row_ok) continue;
                    const int64_t rem_cols = DGT_TILE_FIELD(cx, n, n) - (n0 + ch * 32);
                    const int ncols = rem_cols < 32 ? (int)rem_cols : 32;
                    if constexpr (EPI_MODE == 1) {
                        float* fbase = P.Cf + row + (n0 + ch * 32) * P.ldc;
                        float prevf[32];
                        // read C only when it contributes (a later group, or beta != 0), behind one
                        // warp-uniform branch: with per-element conditions the compiler may issue
                        // the loads anyway (every address is stored to below), and a beta = 0 call
                        // then waits on reads of C it never uses
                        if (g > 0 || P.beta_f != 0.f) {
                            const float ps = g > 0 ? 1.f : P.beta_f;
#pragma unroll
                            for (int c = 0; c < 32; ++c) prevf[c] = c < ncols ? ps * fbase[c * P.ldc] : 0.f;
                        } else {
#pragma unroll
                            for (int c = 0; c < 32; ++c) prevf[c] = 0.f;
                        }
#pragma unroll
                        for (int c = 0; c < 32; ++c)
                            if (c < ncols) fbase[c * P.ldc] = fmaf(P.alpha_f, __uint_as_float(v[c]), prevf[c]);
                        continue;
                    }
                    double prev[32];
                    // ldc, alpha and beta are read at each use, not held in locals: as kernel
                    // parameters they are free operands, while locals made the compiler keep 32
                    // precomputed column addresses live (about 50 more registers, and spills)
#define ldc DGT_TILE_FIELD(cx, ldc, ldc)
#define alpha DGT_TILE_FIELD(cx, alpha, alpha)
#define beta DGT_TILE_FIELD(cx, beta, beta)
                    double* cbase = DGT_TILE_FIELD(cx, C, C) + row + (n0 + ch * 32) * ldc;
                    // C is read only when it contributes (see the FP32 epilogue above); 1.0 * x is
                    // exact, so a later group folds onto C unchanged
                    if (g > 0 || beta != 0.0) {
                        const double ps = g > 0 ? 1.0 : beta;
#pragma unroll
                        for (int c = 0; c < 32; ++c) prev[c] = c < ncols ? ps * cbase[c * ldc] : 0.0;
                    } else {
#pragma unroll
                        for (int c = 0; c < 32; ++c) prev[c] = 0.0;
                    }
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        if (c < ncols) {
                            const int ec = col_exp_s[ch * 32 + c];
                            double t;
                            const double acc_v =
                                (KIND == 0) ? (double)(int32_t)v[c] : (double)__uint_as_float(v[c]);
                            if (e_row == EXP_NONFINITE || ec == EXP_NONFINITE)
                                t = __longlong_as_double(0x7ff8000000000000ll);
                            else
                                t = scale2(acc_v, e_row + ec - 7 * d);
                            cbase[c * ldc] = fma(alpha, t, prev[c]);
                        }
                    }
#undef ldc
#undef alpha
#undef beta
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    if constexpr (PAIR)
                        mbar_arrive_cluster(map_to_rank(acce(b), 0));
                    else
                        mbar_arrive(acce(b));
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if constexpr (PAIR) cluster_sync();  // the leader's MMAs into this CTA's TMEM / smem are done
    tc_fence_after();
    if (warp == 1) {
        if constexpr (PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base), "r"(TMEM_COLS));
        else
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
#undef DGT_TILE_FIELD
}



inline PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
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

// 2D map over the stacked digit planes: [S * rows_pad][k_pad] bytes, box = box_rows x tkb B.
// k_pad_bytes is the row length in bytes (elements * element size).
inline bool make_plane_map(CUtensorMap* map, void* base, int64_t rows_total, int64_t k_pad_bytes, int box_rows,
                           int tkb) {
    auto enc = get_encode();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)k_pad_bytes, (cuuint64_t)rows_total};
    cuuint64_t strides[1] = {(cuuint64_t)k_pad_bytes};
    cuuint32_t box[2] = {(cuuint32_t)tkb, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, tkb == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}


}  // namespace oz
}  // namespace dgt
