// Types shared by the two FP64 emulation schemes' grouped passes (ozaki.cu, ozaki2.cu):
// the per-operand pre-pass job table, and the CRT scheme's modulus tables and reconstruction
// jobs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "dgt_internal.cuh"

namespace dgt {
namespace oz {

// One operand of a grouped pre-pass: a job owns a contiguous range of the launch's blocks,
// found by binary search on the jobs' first block.
struct SplitJob {
    const double* X;
    int64_t ld, MN, K, mn_pad, k_pad;
    unsigned long long* amax;
    int32_t* exps;
    void* planes;
    int32_t kcontig;
    int32_t amax_bx;      // amax blocks along mn (MN-contiguous jobs: times amax_by along K)
    int32_t amax_by;
    int32_t split_bx;     // split blocks along mn (times k_pad / 32 along K)
    int64_t amax_begin;   // first block of this job in the amax launch
    int64_t split_begin;  // first block of this job in the split launch
    int32_t bits;         // CRT scheme: sigma of this operand (scaled rows / columns have 2-norm <= 2^sigma)
    int32_t unused;
    unsigned long long* qn;  // CRT scheme: integer 2-norm bounds per row (see qnorm_*)
    // Row stride of the planes (the product's padded K).  A product whose K is the
    // concatenation of several pieces (K-segments) has one job per piece: planes then points
    // at the piece's first column, K / k_pad are the piece's, and every piece's job updates
    // the row's amax and norm bound with atomics.
    int64_t plane_ld;
};
constexpr int AMAX_KCHUNK = 64;  // K rows per block of the MN-contiguous amax (fills the GPU)

__device__ __forceinline__ int find_job(const SplitJob* __restrict__ jobs, int njobs, int64_t blk, bool split) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int64_t b0 = split ? jobs[mid].split_begin : jobs[mid].amax_begin;
        if (b0 <= blk)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

}  // namespace oz

namespace oz2 {

constexpr int MAX_MODULI = 20, MIN_MODULI = 8;
constexpr int MAX_NW = 5;     // 32-bit limbs of W_p and P (P < 2^160)
constexpr int SPLIT_BITS = 79;  // scaled operands are integers of magnitude below 2^79

// Residues of Y = rn(a 2^s) modulo p, in integers.  The norm rule keeps |Y| <= 2^sigma +
// sqrt(k)/2 < 2^78 (sigma <= 77 for 20 moduli).  Y is taken as yh 2^40 + yl with
// yh = rn(y 2^-40) and yl = rn(y - yh 2^40), |yh|, |yl| <= 2^39 (y - yh 2^40 is exact in
// FP64, and yh 2^40 is an even integer, so the two roundings give rn(y) with its tie
// rule).  Both are cut into 20-bit chunks, x0 = yl mod 2^20, x1 = yl >> 20, x2 = yh mod 2^20,
// x3 = yh >> 20 (arithmetic shifts: |x1|, |x3| <= 2^19), and with c20, c40, c60 = 2^20, 2^40,
// 2^60 mod p in the symmetric range (|c| <= 127; 0 for p = 256)
// t = x3 c60 + x2 c40 + x1 c20 + x0 is congruent to Y with |t| < 127 2^21 + 2^20 < 2^28.
// n = t + floor(p/2) + 2^21 p then lies in (0, 2^30), and with magic = floor(2^38 / p) + 1 =
// 2^38 / p + e (0 < e <= 1), floor(n magic / 2^38) = floor(n / p) because
// n e / 2^38 < 2^30 / 2^38 <= 1 / p (p <= 256).  One 32 x 32 -> 64-bit multiply-add gives
// n magic = t magic + bias.  r = t - floor(n / p) p is the symmetric residue
// ((Y + floor(p/2)) mod p) - floor(p/2) minus 2^21 p, a multiple of 256, so the low byte of r
// is the symmetric residue as int8.
//
// The first nfp moduli take the same residue through the FP64 pipe instead (the integer pipe
// is the split's bound): t = fma(yh, c40, yl) is exact (|t| < 2^39 127 + 2^39 < 2^47),
// q = rint(t / p) from one FMA with fl(1/p) and the round-to-integer constant 1.5 2^52
// (|t / p| < 2^40, so the product is within 2^-12 of t / p, while t / p lies at least
// 1 / (2p) >= 2^-9 from a half-integer for odd p; for p = 256 the product is exact and a tie
// gives r = +-128), and r = t - q p is taken in 32-bit integers from the low words of the
// exact t + 1.5 2^52 and q + 1.5 2^52 (the byte needs r mod 256 only).  For odd p, r is the
// symmetric residue; for p = 256 its byte is the integer path's 0x80 at a tie: the planes are
// the same bytes either way.  At 16384^2, 14 moduli, both operands' amax + norm bound + split
// took 7.0-7.4 ms with every modulus on the integer path, 5.6 with 9 on the FP64 path and 5.4
// with all of them (the 256-product grouped pass at 15 moduli: 15.8 and 15.2 ms), so every
// modulus takes the FP64 path; the integer path stays for builds that set a smaller count.
#ifndef DGT_SPLIT_FP64_MODULI
#define DGT_SPLIT_FP64_MODULI 20
#endif
struct ModTable {
    int32_t p[MAX_MODULI];
    int32_t c20[MAX_MODULI], c40[MAX_MODULI], c60[MAX_MODULI];  // 2^20, 2^40, 2^60 mod p, symmetric
    int32_t magic[MAX_MODULI];                                 // floor(2^38 / p) + 1 (< 2^31 for p > 128)
    long long bias[MAX_MODULI];                                // (floor(p/2) + 2^21 p) magic
    double c40d[MAX_MODULI], invp[MAX_MODULI];                 // the FP64 path's c40 and fl(1/p)
    int32_t nfp;                                               // moduli [0, nfp) take the FP64 path
};
// Residue split geometry: a block of 128 threads covers RES_ROWS rows (mn) and RES_KSPAN
// consecutive kk, one 32-byte sector of every plane row; RES_TPR threads share a row, each
// turning RES_ELEMS consecutive kk into bytes.
constexpr int RES_KSPAN = 32;
constexpr int RES_TPR = 4;
constexpr int RES_ELEMS = RES_KSPAN / RES_TPR;
constexpr int RES_ROWS = 128 / RES_TPR;

struct CrtConst {
    int32_t n;
    uint32_t W[MAX_MODULI][MAX_NW];
    uint32_t P[MAX_NW + 1];
    double kq[MAX_NW + 1];                      // 2^(32 l) / P: X / P ~ sum_l x_l kq_l
    double Wd[MAX_MODULI][MAX_NW];              // W as doubles (exact: every limb < 2^32)
    // the FP64 reconstruction (at most F3_MAX moduli): W and P in three 41-bit limbs as
    // doubles, and fl(2^(41 l) / P)
    double Wf[MAX_MODULI][3];
    double Pf[3], Kf[3];
    // the FP64 limb sums with an integer finish (F3_MAX < n <= F4_MAX): W and P in four 40-bit
    // limbs as doubles, and fl(2^(40 l) / P)
    double Wf4[MAX_MODULI][4];
    double Pf4[4], Kf4[4];
};
constexpr int F3_MAX = 15;  // 15 terms r W_l < 2^49 sum below 2^53; P < 2^123 for 15 moduli
// 20 terms r W_l < 2^48 sum below 2^53; P < 2^160 for 20 moduli.  A build with
// DGT_RECON_F4 = 0 runs the integer limb path above 15 moduli instead (same doubles).
#ifndef DGT_RECON_F4
#define DGT_RECON_F4 1
#endif
constexpr int F4_MAX = DGT_RECON_F4 ? 20 : 0;
// Up to F3_MAX moduli: 0 rounds C' with the correctly rounded three-term FP64 sum
// (crt_value_f3), 1 in integers as above 15 moduli (crt_value_fi); the same doubles either way.
// Measured on one box, alternating builds: 16384^3 at 14 moduli 53.3-53.9 ms per call with the
// FP64 sum against 54.9-55.9 with the integer rounding, the 256-product grouped pass at 15
// moduli 15.4-15.5 against 15.7-15.9 ms.
#ifndef DGT_RECON_F3_INT
#define DGT_RECON_F3_INT 0
#endif

// One product of a grouped reconstruction: its residue planes, exponents, scaling and output;
// it owns threads [thread_begin, thread_begin + ceil(m/4) n) of the launch.  count > 1 makes
// it the lead of a stack group: the count - 1 jobs after it (same m, n, C) are further stacks
// of the same output, own no threads (their thread_begin is the next lead's), and the lead's
// threads write C = (alpha v + beta C) + alpha_1 v_1 + alpha_2 v_2 + ... in that order.
struct CrtJob {
    const uint8_t* res;
    int64_t res_ld, res_plane, m, n;
    const int32_t* row_exp;
    const int32_t* col_exp;
    double alpha, beta;
    double* C;
    int64_t ldc;
    int32_t bits, count;  // bits: sigma_A + sigma_B (the reconstruction's shift is e + f - bits)
    int64_t thread_begin;
};

// host helpers (ozaki2.cu)
int sigma_sum_for(int nmod, int64_t k);  // sigma_A + sigma_B (2-norm bound exponents of rows / columns)
int limbs_for(int nmod);             // 32-bit limbs of P
void crt_constants(int nmod, CrtConst& cc, ModTable& mt);
cudaError_t launch_qnorm_grouped(cudaStream_t s, const oz::SplitJob* jobs, int njobs, int64_t blocks);
cudaError_t launch_split_residues_grouped(cudaStream_t s, const oz::SplitJob* jobs, int njobs, int64_t blocks,
                                          int nmod, const ModTable& mt);
cudaError_t launch_crt_grouped(cudaStream_t s, const CrtJob* jobs, int njobs, int64_t threads, const CrtConst& cc,
                               int nmod);

}  // namespace oz2
// CRT product pieces (ozaki2.cu), for callers that split op(A) once and run op(B) in column
// panels (dgt_dgemm_host): shape and constants of one product (K <= 65536), the workspace
// carve (bytes only when ws is null), one operand's amax + residue split, and the residue
// GEMM + reconstruction of one op(B) panel.
struct Oz2Shape {
    int nmod, sa, sb, variant;  // sa, sb: sigma of op(A) rows and op(B) columns
    bool pair, dyn;             // CTA-pair kernel; dynamic (tile, modulus) unit order
    int64_t m, k, m_pad, n_pad, k_pad;
    oz2::CrtConst cc;
    oz2::ModTable mt;
};
struct Oz2Work {
    size_t bytes = 0;
    int8_t* planesA = nullptr;
    int8_t* planesB = nullptr;
    unsigned long long* amaxA = nullptr;
    unsigned long long* amaxB = nullptr;
    unsigned long long* qnA = nullptr;
    unsigned long long* qnB = nullptr;
    int32_t* expA = nullptr;
    int32_t* expB = nullptr;
    uint8_t* res = nullptr;
    int32_t* sched = nullptr;  // unit counter of the residue GEMM's dynamic order
};
dgt_status ozaki2_shape(dgt_context* h, int64_t m, int64_t n, int64_t k, int nmod, Oz2Shape& sh);
Oz2Work ozaki2_carve(const Oz2Shape& sh, int64_t n, int64_t n_pad, void* ws);
int64_t ozaki2_n_pad(int64_t n);  // op(B) columns padded to the GEMM's tile width
// plane_rows: rows between the operand's modulus planes (0: mn_pad), for a panel written into
// a larger operand's planes (planes then points at the panel's first row of plane 0).
dgt_status ozaki2_split(dgt_context* h, cudaStream_t s, const Oz2Shape& sh, int sigma, const double* X, int64_t ld,
                        int64_t MN, int64_t mn_pad, bool kcontig, unsigned long long* amax, unsigned long long* qn,
                        int32_t* exps, int8_t* planes, int64_t plane_rows = 0);
// The residue GEMM alone (planes strided as for ozaki2_split's plane_rows; spans are the rows
// addressable from each planes pointer) and the reconstruction alone.
dgt_status ozaki2_residue_gemm(dgt_context* h, cudaStream_t s, const Oz2Shape& sh, int64_t n, int64_t n_pad,
                               const int8_t* planesA, const int8_t* planesB, uint8_t* res, int32_t* sched,
                               int64_t a_rows = 0, int64_t a_span = 0, int64_t b_rows = 0, int64_t b_span = 0);
dgt_status ozaki2_reconstruct(dgt_context* h, cudaStream_t s, const Oz2Shape& sh, int64_t n, int64_t n_pad,
                              const uint8_t* res, const int32_t* expA, const int32_t* expB, double alpha, double beta,
                              double* C, int64_t ldc);
dgt_status ozaki2_gemm_crt(dgt_context* h, cudaStream_t s, const Oz2Shape& sh, int64_t n, int64_t n_pad,
                           const int8_t* planesA, const int32_t* expA, const int8_t* planesB, const int32_t* expB,
                           uint8_t* res, double alpha, double beta, double* C, int64_t ldc,
                           int32_t* sched = nullptr);

}  // namespace dgt
