// FP64-accurate GEMM by the Chinese remainder theorem over INT8 residues (Ozaki scheme II:
// Ozaki, Uchino, Imamura 2025, "Ozaki Scheme II: A GEMM-oriented emulation of
// floating-point matrix multiplication using an integer modular technique").
//
//   1. Scale: row i of op(A) gets s_i = sigma - g_i, where 2^g_i bounds the row's 2-norm;
//      A'_ik = rn(a_ik 2^s_i) (rounded to nearest even) is an integer and the row's 2-norm is
//      at most 2^sigma + sqrt(k)/2 (so every entry is below 2^78); columns of op(B) likewise.  By Cauchy-Schwarz every |(A'B')_ij|
//      is below (P/2)(1 - 2^-20) for sigma_A + sigma_B from sigma_sum_for (op(A) takes the
//      odd bit when the sum is odd).  Scaling by the norm instead of
//      the max spends the integer range where the row's mass is: rows with a few large
//      entries among many small ones keep more bits.
//   2. Residues: for N pairwise coprime moduli p <= 256 (P = prod p),
//      A' mod p and B' mod p in the symmetric range [-(p/2), (p-1)/2] are INT8 planes.
//   3. Multiply: (A' mod p)(B' mod p) is exact in INT32 (|sum| <= k 128^2 < 2^31) on the
//      tcgen05 INT8 tensor cores -- one GEMM per modulus, N in all -- and its epilogue keeps
//      only the residue of each element modulo p (one byte).
//   4. Reconstruct: C'_ij = sum_p r_p W_p mod P (W_p = (P/p) ((P/p)^-1 mod p)), taken in
//      the symmetric range, equals (A'B')_ij exactly; it is rounded once to FP64 (correctly)
//      and scaled by 2^-(s_i + t_j).  C = alpha C' + beta_C C.
//
// Entries of a scaled row are not capped below its norm bound: on heavy-tailed rows the
// largest entries exceed 2^53 (they are integers already) and the small ones keep their
// bits down to 2^0, so every added modulus still buys about 4 bits per operand.
// Against the slice scheme (ozaki.cu), N GEMMs replace S(S+1)/2 digit products for the
// same number of operand bits (N = 17 moduli: sigma = 65-66 bits at K <= 16384, versus 36
// products for S = 8 slices of 7 bits), and the output is read and written once instead of
// once per flush group.  The FLOP count reported for this path is 2*M*N*K.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <vector>

#include "crt.cuh"
#include "dgt_internal.cuh"
#include "tc_engine.cuh"

namespace dgt {
namespace oz2 {

// Pairwise coprime, largest first (greedy from 256 down).
constexpr int kModuli[MAX_MODULI] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                     223, 217, 211, 199, 197, 193, 191, 181, 179, 173};
constexpr bool moduli_in_split_range() {  // the residue split's magic divide needs 128 < p <= 256
    for (int p : kModuli)
        if (p <= 128 || p > 256) return false;
    return true;
}
static_assert(moduli_in_split_range(), "CRT moduli must lie in (128, 256]");

// ---- host: CRT constants in 32-bit limbs ------------------------------------------------------
using Big = std::vector<uint32_t>;  // little-endian limbs

static void big_mul_small(Big& a, uint32_t m) {
    uint64_t c = 0;
    for (auto& x : a) {
        const uint64_t t = (uint64_t)x * m + c;
        x = (uint32_t)t;
        c = t >> 32;
    }
    if (c) a.push_back((uint32_t)c);
}

static uint32_t big_div_small(Big& a, uint32_t d) {  // a /= d, returns a mod d
    uint64_t r = 0;
    for (size_t i = a.size(); i-- > 0;) {
        const uint64_t cur = (r << 32) | a[i];
        a[i] = (uint32_t)(cur / d);
        r = cur % d;
    }
    while (a.size() > 1 && a.back() == 0) a.pop_back();
    return (uint32_t)r;
}

static uint32_t inv_mod(uint32_t a, uint32_t p) {  // a^-1 mod p (gcd(a, p) = 1)
    int64_t t = 0, nt = 1, r = p, nr = a % p;
    while (nr) {
        const int64_t q = r / nr;
        std::swap(t, nt);
        nt -= q * t;
        std::swap(r, nr);
        nr -= q * r;
    }
    return (uint32_t)(t < 0 ? t + p : t);
}

static double log2_product(int n) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += std::log2((double)kModuli[i]);
    return s;
}

// Norm scaling.  Row i of op(A) is scaled by 2^s_i with s_i = sigma - g_i: 2^g_i bounds the
// row's 2-norm (g_i from the integer bound of qnorm_*), so every scaled row has 2-norm
// <= 2^sigma; columns of op(B) likewise.  After rounding to nearest, ||A'_i|| <= 2^sigma + sqrt(k)/2, and
// by Cauchy-Schwarz |C'_ij| <= (2^sigma + sqrt(k)/2)^2.  sigma is the largest integer keeping
// that below (P/2)(1 - 2^-20), which the reconstruction's exact quotient needs (the sqrt(k)/2
// terms are below 2^-40 of 2^sigma for every sigma used, well inside the margin).
int sigma_sum_for(int n, int64_t k) {
    // the largest s with (2^ceil(s/2) + r)(2^floor(s/2) + r) < (P / 2)(1 - 2^-20), r = sqrt(k) / 2,
    // checked in the log domain with a 1e-9 margin (op(A) takes ceil(s/2), op(B) floor(s/2))
    const double t = log2_product(n) - 1.0 + std::log2(1.0 - std::ldexp(1.0, -20));
    const double r = std::sqrt((double)std::max<int64_t>(k, 1)) / 2.0;
    int s = (int)std::floor(t);
    while (s > 0) {
        const double a = std::ldexp(1.0, (s + 1) / 2), b = std::ldexp(1.0, s / 2);
        if (std::log2((a + r) * (b + r)) < t - 1e-9) break;
        --s;
    }
    return s;
}

// Limbs of W_p and P for n moduli (P < 2^(32 nw)).
int limbs_for(int n) { return (int)std::ceil(log2_product(n) / 32.0); }

void crt_constants(int n, CrtConst& cc, ModTable& mt) {
    cc = CrtConst{};
    mt = ModTable{};
    cc.n = n;
    Big P{1};
    for (int i = 0; i < n; ++i) big_mul_small(P, (uint32_t)kModuli[i]);
    for (int i = 0; i < n; ++i) {
        const uint32_t p = (uint32_t)kModuli[i];
        mt.p[i] = (int32_t)p;
        auto sym = [p](unsigned long long v) { return (int32_t)(v > p / 2 ? (long long)v - p : (long long)v); };
        mt.c20[i] = sym((1ull << 20) % p);
        mt.c40[i] = sym((1ull << 40) % p);
        mt.c60[i] = sym((1ull << 60) % p);
        mt.magic[i] = (int32_t)((1ull << 38) / p + 1);
        mt.bias[i] = ((long long)(p >> 1) + ((long long)p << 21)) * mt.magic[i];
        mt.c40d[i] = (double)mt.c40[i];
        mt.invp[i] = 1.0 / (double)p;
        Big M = P;
        big_div_small(M, p);  // M = P / p
        Big Mm = M;
        const uint32_t m_mod = big_div_small(Mm, p);
        big_mul_small(M, inv_mod(m_mod, p));  // W = M * (M^-1 mod p) < P
        for (int l = 0; l < MAX_NW; ++l) {
            cc.W[i][l] = l < (int)M.size() ? M[l] : 0;
            cc.Wd[i][l] = (double)cc.W[i][l];
        }
    }
    mt.nfp = std::min(n, DGT_SPLIT_FP64_MODULI);
    for (int l = 0; l <= MAX_NW; ++l) cc.P[l] = l < (int)P.size() ? P[l] : 0;
    double pd = 0;
    for (int l = MAX_NW; l >= 0; --l) pd = pd * 4294967296.0 + (double)cc.P[l];
    for (int l = 0; l <= MAX_NW; ++l) cc.kq[l] = std::ldexp(1.0, 32 * l) / pd;
    // 41-bit limbs (bits [41 l, 41 l + 41)) for the FP64 reconstruction, 40-bit ones for the
    // FP64 limb sums with the integer finish
    auto limb = [](const Big& x, int l, int width) {
        uint64_t v = 0;
        for (int b = 0; b < width; ++b) {
            const int bit = width * l + b, w = bit / 32;
            if (w < (int)x.size() && ((x[w] >> (bit % 32)) & 1u)) v |= 1ull << b;
        }
        return (double)v;
    };
    auto limb41 = [&](const Big& x, int l) { return limb(x, l, 41); };
    for (int i = 0; i < n; ++i) {
        Big M = P;
        big_div_small(M, (uint32_t)kModuli[i]);
        Big Mm = M;
        const uint32_t m_mod = big_div_small(Mm, (uint32_t)kModuli[i]);
        big_mul_small(M, inv_mod(m_mod, (uint32_t)kModuli[i]));  // W_i, as above
        for (int l = 0; l < 3; ++l) cc.Wf[i][l] = limb41(M, l);
        for (int l = 0; l < 4; ++l) cc.Wf4[i][l] = limb(M, l, 40);
    }
    for (int l = 0; l < 3; ++l) {
        cc.Pf[l] = limb41(P, l);
        cc.Kf[l] = std::ldexp(1.0, 41 * l) / pd;
    }
    for (int l = 0; l < 4; ++l) {
        cc.Pf4[l] = limb(P, l, 40);
        cc.Kf4[l] = std::ldexp(1.0, 40 * l) / pd;
    }
}

// ---- device: row norms ---------------------------------------------------------------------------
// Upper bound of a row's squared 2-norm relative to its max exponent e (max |x| < 2^e):
// q = sum_k ceil(|x| 2^(20-e))^2, each term an integer <= 2^40 and >= (|x| 2^(20-e))^2.
// Terms are added in FP64 in runs of at most 4096 (partial sums below 2^52: exact), each run
// converted to an integer and summed in integers, so the bound and every result derived from
// it are deterministic; ||x||_2 <= 2^(e-20) sqrt(q).  2^(20-e) is one double for e >= -1002
// (the general scaling otherwise); a product that lands below the normal range only rounds
// terms of size < 2^-2000, far inside the reconstruction's 2^-20 margin.
struct QScale {
    double f;
    int sh;
    bool direct;
};
__device__ __forceinline__ QScale qscale(int e) {
    QScale q;
    q.sh = 20 - e;
    q.direct = q.sh <= 1023;
    q.f = q.direct ? oz::pow2i(max(q.sh, -1022)) : 0.0;
    return q;
}
__device__ __forceinline__ double sq_term(double x, const QScale& q) {
    const double c = ceil(q.direct ? fabs(x) * q.f : oz::scale2(fabs(x), q.sh));
    return c * c;  // exact: c <= 2^20
}

// MN-contiguous operand (element (mn, kk) at X[mn + kk ld]): thread per mn, K in chunks of
// at most 64 across blocks, integer atomic sums (q zeroed by the caller).
__device__ __forceinline__ void qnorm_mn_block(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                               int kchunk, const unsigned long long* __restrict__ amax,
                                               unsigned long long* __restrict__ q, int64_t bx, int64_t by) {
    const int64_t mn = bx * blockDim.x + threadIdx.x;
    if (mn >= MN) return;
    const unsigned long long am = amax[mn];
    const int e = oz::exponent_of_max(am);
    if (am == 0ull || e == oz::EXP_NONFINITE) return;
    const QScale qs = qscale(e);
    const int64_t k0 = by * kchunk, k1 = min(K, k0 + kchunk);
    double acc = 0.0;
    for (int64_t kk = k0; kk < k1; ++kk) acc += sq_term(X[mn + kk * ld], qs);
    if (acc != 0.0) atomicAdd(q + mn, (unsigned long long)acc);
}

// K-contiguous operand (element (mn, kk) at X[kk + mn ld]): warp per mn; each lane's run is
// at most ceil(K / 32) <= 4096 terms.
// atomic: the row may have other pieces (q zeroed by the caller), so the sum goes in by atomicAdd.
__device__ __forceinline__ void qnorm_k_block(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                              const unsigned long long* __restrict__ amax,
                                              unsigned long long* __restrict__ q, int64_t bx, bool atomic = false) {
    const int64_t mn = bx * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (mn >= MN) return;
    const unsigned long long am = amax[mn];
    const int e = oz::exponent_of_max(am);
    double acc = 0.0;
    if (am != 0ull && e != oz::EXP_NONFINITE) {
        const QScale qs = qscale(e);
        const double* row = X + mn * ld;
        for (int64_t kk = lane; kk < K; kk += 32) acc += sq_term(row[kk], qs);
    }
    unsigned long long t = (unsigned long long)acc;
#pragma unroll
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) {
        if (!atomic)
            q[mn] = t;
        else if (t)
            atomicAdd(q + mn, t);
    }
}

__global__ void qnorm_mn_contig(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K, int kchunk,
                                const unsigned long long* __restrict__ amax, unsigned long long* __restrict__ q) {
    qnorm_mn_block(X, ld, MN, K, kchunk, amax, q, blockIdx.x, blockIdx.y);
}
__global__ void qnorm_k_contig(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                               const unsigned long long* __restrict__ amax, unsigned long long* __restrict__ q) {
    qnorm_k_block(X, ld, MN, K, amax, q, blockIdx.x);
}
// Every operand of a grouped call, on the amax launch's block layout.
__global__ void __launch_bounds__(256) qnorm_grouped(const oz::SplitJob* __restrict__ jobs, int njobs) {
    const int64_t blk = blockIdx.x;
    const oz::SplitJob& J = jobs[oz::find_job(jobs, njobs, blk, false)];
    const int64_t local = blk - J.amax_begin;
    if (J.kcontig)
        qnorm_k_block(J.X, J.ld, J.MN, J.K, J.amax, J.qn, local, true);
    else
        qnorm_mn_block(J.X, J.ld, J.MN, J.K, oz::AMAX_KCHUNK, J.amax, J.qn, local % J.amax_bx, local / J.amax_bx);
}

// Scale of row mn: exps[mn] = sigma - s = g with s = sigma - g (sigma = sigma_A for rows of
// op(A), sigma_B for columns of op(B); see sigma_sum_for); EXP_NONFINITE for a row with an
// infinite or NaN element.
__device__ __forceinline__ int row_scale_exp(unsigned long long am, unsigned long long qv, int sigma, int& s) {
    const int e = oz::exponent_of_max(am);
    if (e == oz::EXP_NONFINITE) return e;
    if (am == 0ull || qv == 0ull) {
        s = 0;
        return sigma;
    }
    const int h = (64 - __clzll((long long)(qv - 1ull)) + 1) >> 1;  // 2^h >= sqrt(qv)
    const int g = e - 20 + h;
    s = sigma - g;
    return g;
}

// ---- device: residue planes ----------------------------------------------------------------------
// Plane j holds (A' mod p_j) in the symmetric range as int8 at [j][mn][kk] (K-major, row
// stride pld >= k_pad, mn_pad rows, zero padded to k_pad; pld > k_pad for one piece of a
// concatenated K), planes pstride bytes apart (>= mn_pad pld; more for a panel of a larger
// operand's planes).  A thread produces RES_ELEMS consecutive kk of one
// mn; the RES_TPR adjacent lanes of a row write one whole 32-byte sector per plane together
// (lanes that wrote parts of a sector each made L2 fetch the sector from DRAM first).  The
// seg == 0, by == 0 threads also write exps[mn].
template <bool K_CONTIG>
__device__ __forceinline__ void residue_block(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                              int64_t mn_pad, int64_t k_pad, int64_t pld, int64_t pstride, int nmod,
                                              int sigma, const unsigned long long* __restrict__ amax,
                                              const unsigned long long* __restrict__ qn, int32_t* __restrict__ exps,
                                              int8_t* __restrict__ planes, const ModTable& mt, int64_t bx,
                                              int64_t by) {
    constexpr int E = RES_ELEMS;
    static_assert(E == 8 || E % 16 == 0, "residue split: RES_ELEMS must be 8 or a multiple of 16");
    const int row = threadIdx.x / RES_TPR, seg = threadIdx.x % RES_TPR;
    const int64_t mn = bx * RES_ROWS + row;
    const int64_t k0 = by * RES_KSPAN + seg * E;
    // MN-contiguous operand: the block's RES_ROWS x RES_KSPAN tile comes in through shared
    // memory, every warp load one kk over RES_ROWS consecutive mn (a thread's own kk run would
    // touch one 8-byte word per row); rows of RES_ROWS + 1 doubles keep the reads at two
    // wavefronts per warp
    constexpr int TLD = RES_ROWS + 1;
    __shared__ double tile[K_CONTIG ? 1 : RES_KSPAN * TLD];
    if constexpr (!K_CONTIG) {
        static_assert(128 % RES_ROWS == 0 && RES_KSPAN % (128 / RES_ROWS) == 0, "residue split: tile shape");
        constexpr int KSTEP = 128 / RES_ROWS;
        const int lm = threadIdx.x % RES_ROWS, kq = threadIdx.x / RES_ROWS;
        const int64_t tm = bx * RES_ROWS + lm, tk0 = by * RES_KSPAN;
#pragma unroll
        for (int i = 0; i < RES_KSPAN / KSTEP; ++i) {
            const int kl = kq + KSTEP * i;
            tile[kl * TLD + lm] = (tm < MN && tk0 + kl < K) ? X[tm + (tk0 + kl) * ld] : 0.0;
        }
        __syncthreads();
    }
    if (mn >= mn_pad) return;
    int e = 0, sc = 0;  // sc: this row's scale exponent s
    if (mn < MN) {
        e = row_scale_exp(amax[mn], qn[mn], sigma, sc);
        if (by == 0 && seg == 0) exps[mn] = e;
    }
    const bool live = (mn < MN) && (e != oz::EXP_NONFINITE);
    // 2^sc as one double when it is one (the product is then exact, or below 2^-1022 where
    // it rounds to the integer 0 either way); the general scaling otherwise
    const bool direct = sc >= -1022 && sc <= 1023;
    const double fsc = direct ? oz::pow2i(sc) : 0.0;
    const int64_t plane = pstride;
    int8_t* out = planes + mn * pld + k0;
    if (!live || k0 >= K) {  // padding (or a non-finite row): zero residues, no arithmetic
#pragma unroll 4
        for (int j = 0; j < nmod; ++j, out += plane) {
            if constexpr (E % 16 == 0) {
#pragma unroll
                for (int q = 0; q < E / 16; ++q) reinterpret_cast<uint4*>(out)[q] = make_uint4(0u, 0u, 0u, 0u);
            } else {
                *reinterpret_cast<uint2*>(out) = make_uint2(0u, 0u);
            }
        }
        return;
    }
    // Y = x3 2^60 + x2 2^40 + x1 2^20 + x0 (crt.cuh ModTable): x0, x2 in [0, 2^20), |x1|, |x3| <= 2^19
    int32_t x0[E], x1[E], x2[E], x3[E];
    double yhd[E], yld[E];  // Y = yh 2^40 + yl as doubles, for the FP64 path
#pragma unroll
    for (int i = 0; i < E; ++i) {
        const int64_t kk = k0 + i;
        double a = 0.0;
        if (live && kk < K) a = K_CONTIG ? X[kk + mn * ld] : tile[(seg * E + i) * TLD + row];
        // y = a 2^sc exactly; Y = rn(y) = yh 2^40 + yl, |yh|, |yl| <= 2^39
        const double y = live ? (direct ? a * fsc : oz::scale2(a, sc)) : 0.0;
        const double yh = rint(y * 0x1p-40);
        const double yl = rint(fma(-yh, 0x1p40, y));  // the second rounding: Y = yh 2^40 + yl
        yhd[i] = yh;
        yld[i] = yl;
        const long long hi = __double2ll_rn(yh), lo = __double2ll_rn(yl);
        x0[i] = (int32_t)(lo & 0xfffff);
        x1[i] = (int32_t)(lo >> 20);
        x2[i] = (int32_t)(hi & 0xfffff);
        x3[i] = (int32_t)(hi >> 20);
    }
    constexpr double RINT = 6755399441055744.0;  // 1.5 2^52: adding it rounds to an integer
    const int nfp = min(mt.nfp, nmod);
    for (int j = 0; j < nfp; ++j, out += plane) {
        const double c40 = mt.c40d[j], ip = mt.invp[j];
        const int32_t p = mt.p[j];
        uint32_t w[E / 4];
#pragma unroll
        for (int q = 0; q < E / 4; ++q) {
            int32_t r[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = 4 * q + u;
                const double t = fma(yhd[i], c40, yld[i]);  // = Y mod p, |t| < 2^47, exact
                // t + 1.5 2^52 and 1.5 2^52 + rint(t / p) are exact and carry t and q in their
                // low words (mod 2^32); only the low byte of r = t - q p is kept, so the low
                // words suffice
                const int32_t tl = __double2loint(t + RINT), ql = __double2loint(fma(t, ip, RINT));
                r[u] = tl - ql * p;
            }
            w[q] = __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
        }
        if constexpr (E % 16 == 0) {
#pragma unroll
            for (int q = 0; q < E / 16; ++q)
                reinterpret_cast<uint4*>(out)[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
        } else {
            *reinterpret_cast<uint2*>(out) = make_uint2(w[0], w[1]);
        }
    }
    for (int j = nfp; j < nmod; ++j, out += plane) {
        const int32_t p = mt.p[j], c20 = mt.c20[j], c40 = mt.c40[j], c60 = mt.c60[j], mg = mt.magic[j];
        const long long bias = mt.bias[j];
        uint32_t w[E / 4];
#pragma unroll
        for (int q = 0; q < E / 4; ++q) {
            int32_t r[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = 4 * q + u;
                const int32_t t = x3[i] * c60 + x2[i] * c40 + x1[i] * c20 + x0[i];  // = Y mod p, |t| < 2^28
                const int32_t qt = (int32_t)((unsigned long long)((long long)t * mg + bias) >> 38);
                r[u] = t - qt * p;  // low byte: the symmetric residue
            }
            w[q] = __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
        }
        if constexpr (E % 16 == 0) {
#pragma unroll
            for (int q = 0; q < E / 16; ++q)
                reinterpret_cast<uint4*>(out)[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
        } else {
            *reinterpret_cast<uint2*>(out) = make_uint2(w[0], w[1]);
        }
    }
}

template <bool K_CONTIG>
__global__ void __launch_bounds__(128) split_residues(const double* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                                      int64_t mn_pad, int64_t k_pad, int64_t pstride, int nmod,
                                                      int sigma, const unsigned long long* __restrict__ amax,
                                                      const unsigned long long* __restrict__ qn,
                                                      int32_t* __restrict__ exps, int8_t* __restrict__ planes,
                                                      const __grid_constant__ ModTable mt) {
    residue_block<K_CONTIG>(X, ld, MN, K, mn_pad, k_pad, k_pad, pstride, nmod, sigma, amax, qn, exps, planes, mt,
                            blockIdx.x, blockIdx.y);
}

// Every operand of a grouped call in one launch (job table as for the digit split).
__global__ void __launch_bounds__(128) split_residues_grouped(const oz::SplitJob* __restrict__ jobs, int njobs,
                                                              int nmod, const __grid_constant__ ModTable mt) {
    const int64_t blk = blockIdx.x;
    const oz::SplitJob& J = jobs[oz::find_job(jobs, njobs, blk, true)];
    const int64_t local = blk - J.split_begin;
    const int64_t bx = local % J.split_bx, by = local / J.split_bx;
    if (J.kcontig)
        residue_block<true>(J.X, J.ld, J.MN, J.K, J.mn_pad, J.k_pad, J.plane_ld, J.mn_pad * J.plane_ld, nmod, J.bits, J.amax, J.qn, J.exps,
                            (int8_t*)J.planes, mt, bx, by);
    else
        residue_block<false>(J.X, J.ld, J.MN, J.K, J.mn_pad, J.k_pad, J.plane_ld, J.mn_pad * J.plane_ld, nmod, J.bits, J.amax, J.qn, J.exps,
                             (int8_t*)J.planes, mt, bx, by);
}

// ---- device: reconstruction -----------------------------------------------------------------------
// x += y (ADD) or x -= y over N 32-bit limbs, one carry chain.
template <int N, bool ADD>
__device__ __forceinline__ void limbs_addsub(uint32_t (&x)[N], const uint32_t (&y)[N]) {
    if constexpr (N == 3) {
        if constexpr (ADD)
        asm("add.cc.u32 %0, %0, %3;\n" "addc.cc.u32 %1, %1, %4;\n" "addc.u32 %2, %2, %5;\n"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2])
            : "r"(y[0]), "r"(y[1]), "r"(y[2]));
        else
        asm("sub.cc.u32 %0, %0, %3;\n" "subc.cc.u32 %1, %1, %4;\n" "subc.u32 %2, %2, %5;\n"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2])
            : "r"(y[0]), "r"(y[1]), "r"(y[2]));
    }
    if constexpr (N == 4) {
        if constexpr (ADD)
        asm("add.cc.u32 %0, %0, %4;\n" "addc.cc.u32 %1, %1, %5;\n" "addc.cc.u32 %2, %2, %6;\n" "addc.u32 %3, %3, %7;\n"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3])
            : "r"(y[0]), "r"(y[1]), "r"(y[2]), "r"(y[3]));
        else
        asm("sub.cc.u32 %0, %0, %4;\n" "subc.cc.u32 %1, %1, %5;\n" "subc.cc.u32 %2, %2, %6;\n" "subc.u32 %3, %3, %7;\n"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3])
            : "r"(y[0]), "r"(y[1]), "r"(y[2]), "r"(y[3]));
    }
    if constexpr (N == 5) {
        if constexpr (ADD)
        asm("add.cc.u32 %0, %0, %5;\n" "addc.cc.u32 %1, %1, %6;\n" "addc.cc.u32 %2, %2, %7;\n" "addc.cc.u32 %3, %3, %8;\n" "addc.u32 %4, %4, %9;\n"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4])
            : "r"(y[0]), "r"(y[1]), "r"(y[2]), "r"(y[3]), "r"(y[4]));
        else
        asm("sub.cc.u32 %0, %0, %5;\n" "subc.cc.u32 %1, %1, %6;\n" "subc.cc.u32 %2, %2, %7;\n" "subc.cc.u32 %3, %3, %8;\n" "subc.u32 %4, %4, %9;\n"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4])
            : "r"(y[0]), "r"(y[1]), "r"(y[2]), "r"(y[3]), "r"(y[4]));
    }
    if constexpr (N == 6) {
        if constexpr (ADD)
        asm("add.cc.u32 %0, %0, %6;\n" "addc.cc.u32 %1, %1, %7;\n" "addc.cc.u32 %2, %2, %8;\n" "addc.cc.u32 %3, %3, %9;\n" "addc.cc.u32 %4, %4, %10;\n" "addc.u32 %5, %5, %11;\n"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5])
            : "r"(y[0]), "r"(y[1]), "r"(y[2]), "r"(y[3]), "r"(y[4]), "r"(y[5]));
        else
        asm("sub.cc.u32 %0, %0, %6;\n" "subc.cc.u32 %1, %1, %7;\n" "subc.cc.u32 %2, %2, %8;\n" "subc.cc.u32 %3, %3, %9;\n" "subc.cc.u32 %4, %4, %10;\n" "subc.u32 %5, %5, %11;\n"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5])
            : "r"(y[0]), "r"(y[1]), "r"(y[2]), "r"(y[3]), "r"(y[4]), "r"(y[5]));
    }
}

// x + y rounded to odd: the exact sum when it is a double, else the neighbour of the exact
// sum (toward zero or away) whose last mantissa bit is 1 -- the round-toward-zero result with
// that bit set.  TwoSum (Knuth) tells exact from inexact.
__device__ __forceinline__ double add_round_odd(double x, double y) {
    const double s = __dadd_rn(x, y);
    const double bb = __dsub_rn(s, x);
    const double e = __dadd_rn(__dsub_rn(x, __dsub_rn(s, bb)), __dsub_rn(y, bb));
    if (e == 0.0) return s;
    return __longlong_as_double(__double_as_longlong(__dadd_rz(x, y)) | 1ll);
}
// a + b + c rounded once to the nearest double (ties to even): Boldo and Melquiond's adder
// ("Emulation of FMA and correctly rounded sums: proved algorithms using rounding to odd",
// IEEE Trans. Computers 57(4), 2008): two TwoSums, the two error terms added with rounding to
// odd, then one rounding to nearest.  Valid for doubles without underflow or overflow.
__device__ __forceinline__ double sum3_rn(double a, double b, double c) {
    const double uh = __dadd_rn(b, c);
    const double ub = __dsub_rn(uh, b);
    const double ul = __dadd_rn(__dsub_rn(b, __dsub_rn(uh, ub)), __dsub_rn(c, ub));
    const double th = __dadd_rn(a, uh);
    const double tb = __dsub_rn(th, a);
    const double tl = __dadd_rn(__dsub_rn(a, __dsub_rn(th, tb)), __dsub_rn(uh, tb));
    return __dadd_rn(th, add_round_odd(tl, ul));
}

// The same value as crt_value, through the FP64 pipe, for at most F3_MAX moduli.  X = S0 +
// S1 2^41 + S2 2^82 with S_l = sum_j r_j w_jl (w_jl the 41-bit limbs of W_j: every term below
// 2^49, the sum below 2^53, exact).  q = round(X / P) from S_l fl(2^(41 l) / P) (X / P < 2^12,
// the estimate within 2^-38, inside the 2^-20 margin), and d_l = S_l - q P_l is exact (both
// below 2^53), so C' = X - q P = d0 + d1 2^41 + d2 2^82 exactly, rounded once by sum3_rn.  The
// scaling then runs on the mantissa and exponent crt_value would hand it, so the result is
// the same double in every case, subnormal results included.
template <int NM>
__device__ __forceinline__ double crt_value_f3(const uint32_t (&rr)[MAX_MODULI], int sel, const CrtConst& cc,
                                               int shift) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int j = 0; j < MAX_MODULI; ++j) {
        if (NM ? j < NM : j < cc.n) {
            const uint32_t r = __byte_perm(rr[j], 0u, 0x4440u + (uint32_t)sel);  // byte sel
            const double rd = __hiloint2double(0x43300000, (int)r) - 4503599627370496.0;
            s0 = fma(rd, cc.Wf[j][0], s0);
            s1 = fma(rd, cc.Wf[j][1], s1);
            s2 = fma(rd, cc.Wf[j][2], s2);
        }
    }
    const double q = rint(fma(s2, cc.Kf[2], fma(s1, cc.Kf[1], s0 * cc.Kf[0])));
    const double d0 = fma(-q, cc.Pf[0], s0), d1 = fma(-q, cc.Pf[1], s1), d2 = fma(-q, cc.Pf[2], s2);
    const double z = sum3_rn(d2 * 0x1p82, d1 * 0x1p41, d0);
    if (z == 0.0) return 0.0;
    // z = m 2^ez with m in [1, 2): hand scale2 the mantissa in [2^63, 2^64) as crt_value does
    const long long bits = __double_as_longlong(z);
    const int ez = (int)((bits >> 52) & 0x7ff) - 1023;
    const double zm = __longlong_as_double((bits & ~(0x7ffll << 52)) | ((long long)(1023 + 63) << 52));
    return oz::scale2(zm, ez - 63 + shift);
}

// The same value as crt_value with the limb sums through the FP64 pipe and the rounding in
// integers: L = 3 limbs of 41 bits (the F3 constants, up to F3_MAX moduli) or L = 4 limbs of
// 40 bits (F3_MAX < n <= F4_MAX).  X = sum_l S_l 2^(B l) with S_l = sum_j r_j w_jl (w_jl the
// B-bit limbs of W_j: every term below 2^(B+8), the sum below 2^53, exact).  q = round(X / P)
// from S_l fl(2^(B l) / P) (X / P < 20 * 255 < 2^13, the estimate within 2^-37, inside the
// 2^-21 margin the norm rule leaves), and d_l = S_l - q P_l is exact (q P_l < 2^53, the
// difference an integer below 2^53).  The d_l become 64-bit integers, carries make the low
// L - 1 digits non-negative (the top one keeps the sign: |C'| < P / 2), and the digits pack
// into three 64-bit words of C' in two's complement.  Its magnitude is rounded exactly as
// crt_value rounds it (top word, the word below, a sticky bit for the rest, one conversion),
// so the result is the same double.
template <int L, int NM>
__device__ __forceinline__ double crt_value_fi(const uint32_t (&rr)[MAX_MODULI], int sel, const CrtConst& cc,
                                               int shift) {
    static_assert(L == 3 || L == 4, "FP64 limb sums: 3 or 4 limbs");
    constexpr int B = L == 3 ? 41 : 40;
    double sl[L];
#pragma unroll
    for (int l = 0; l < L; ++l) sl[l] = 0.0;
#pragma unroll
    for (int j = 0; j < MAX_MODULI; ++j) {
        if (NM ? j < NM : j < cc.n) {
            const uint32_t r = __byte_perm(rr[j], 0u, 0x4440u + (uint32_t)sel);  // byte sel
            const double rd = __hiloint2double(0x43300000, (int)r) - 4503599627370496.0;
#pragma unroll
            for (int l = 0; l < L; ++l) sl[l] = fma(rd, L == 3 ? cc.Wf[j][l] : cc.Wf4[j][l], sl[l]);
        }
    }
    double xq = sl[0] * (L == 3 ? cc.Kf[0] : cc.Kf4[0]);
#pragma unroll
    for (int l = 1; l < L; ++l) xq = fma(sl[l], L == 3 ? cc.Kf[l] : cc.Kf4[l], xq);
    const double q = rint(xq);
    long long d[L];
#pragma unroll
    for (int l = 0; l < L; ++l) d[l] = __double2ll_rn(fma(-q, L == 3 ? cc.Pf[l] : cc.Pf4[l], sl[l]));
    constexpr long long MB = (1ll << B) - 1;
#pragma unroll
    for (int l = 0; l + 1 < L; ++l) {
        d[l + 1] += d[l] >> B;  // arithmetic shift: floor division by 2^B
        d[l] &= MB;
    }
    // C' = sum_l d_l 2^(B l), digits d_0 .. d_(L-2) in [0, 2^B), as three words (the top
    // digit's arithmetic shifts fill the words above it with its sign)
    uint64_t w[3] = {0ull, 0ull, 0ull};
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const int o = B * l, i = o / 64, sh = o % 64;
        w[i] |= (uint64_t)d[l] << sh;
        if (sh > 0 && i + 1 < 3) w[i + 1] |= (uint64_t)(d[l] >> (64 - sh));
        if (l == L - 1 && i + 2 < 3) w[i + 2] = (uint64_t)(d[l] >> 63);
    }
    uint64_t w0 = w[0], w1 = w[1], w2 = w[2];
    const bool neg = d[L - 1] < 0;
    if (neg) {  // magnitude -C' (three-word two's complement negation)
        const uint64_t n0 = ~w0 + 1ull;
        const uint64_t c0 = w0 == 0ull ? 1ull : 0ull;
        const uint64_t n1 = ~w1 + c0;
        const uint64_t c1 = (c0 != 0ull && w1 == 0ull) ? 1ull : 0ull;
        w2 = ~w2 + c1;
        w1 = n1;
        w0 = n0;
    }
    uint64_t hi = w0, lo = 0ull;
    bool sticky = false;
    int ti = 0;
    if (w2 != 0ull) {
        hi = w2;
        lo = w1;
        sticky = w0 != 0ull;
        ti = 2;
    } else if (w1 != 0ull) {
        hi = w1;
        lo = w0;
        ti = 1;
    }
    if (hi == 0ull) return 0.0;
    const int lz = __clzll((long long)hi);
    const uint64_t top64 = lz ? (hi << lz) | (lo >> (64 - lz)) : hi;
    sticky |= (lz ? (lo << lz) : lo) != 0ull;
    const double dv = __ull2double_rn(top64 | (uint64_t)sticky);
    const double mag = oz::scale2(dv, 64 * ti - lz + shift);
    return neg ? -mag : mag;
}

// X = sum_j r_j W_j (NW-limb W, NX = NW + 1 limbs for X < 2^13 P) reduced mod P into the
// symmetric range, rounded to FP64 once (round to nearest even), times 2^shift.  r_j is byte
// `sel` of rr[j]; NM is the modulus count when known at compile time (0: cc.n).  Constant trip
// counts keep every limb in registers.
template <int NW, int NM>
__device__ __forceinline__ double crt_value(const uint32_t (&rr)[MAX_MODULI], int sel, const CrtConst& cc,
                                            int shift) {
    if constexpr (NM != 0 && NM <= F3_MAX) {
        if constexpr (DGT_RECON_F3_INT)
            return crt_value_fi<3, NM>(rr, sel, cc, shift);  // FP64 limb sums, integer rounding
        else
            return crt_value_f3<NM>(rr, sel, cc, shift);  // the FP64 form (same value)
    } else if constexpr (NM != 0 && NM <= F4_MAX) {
        return crt_value_fi<4, NM>(rr, sel, cc, shift);  // FP64 limb sums, integer rounding (same value)
    } else {
    if (NM == 0 && cc.n <= F3_MAX)
        return DGT_RECON_F3_INT ? crt_value_fi<3, 0>(rr, sel, cc, shift) : crt_value_f3<0>(rr, sel, cc, shift);
    constexpr int NX = NW + 1;
    // The low NI limbs accumulate in 64-bit integers, the high ones in FP64, which is exact:
    // r W_l < 2^40 and at most 20 of them sum below 2^45 < 2^53.  Splitting the multiply-adds
    // between the integer and the (otherwise idle) FP64 pipe halves the longest pipe's work.
    constexpr int NI = NW / 2;
    uint64_t acc[NW];
    double accd[NW - NI];
#pragma unroll
    for (int l = 0; l < NW; ++l) acc[l] = 0;
#pragma unroll
    for (int l = 0; l < NW - NI; ++l) accd[l] = 0.0;
#pragma unroll
    for (int j = 0; j < MAX_MODULI; ++j) {
        if (NM ? j < NM : j < cc.n) {
            const uint32_t r = __byte_perm(rr[j], 0u, 0x4440u + (uint32_t)sel);  // byte sel
#pragma unroll
            for (int l = 0; l < NI; ++l) acc[l] += (uint64_t)r * cc.W[j][l];  // < 20 * 2^40
            // r as a double: 2^52 + r has r in its low mantissa bits, then subtract 2^52 (exact)
            const double rd = __hiloint2double(0x43300000, (int)r) - 4503599627370496.0;
#pragma unroll
            for (int l = NI; l < NW; ++l) accd[l - NI] = fma(rd, cc.Wd[j][l], accd[l - NI]);
        }
    }
#pragma unroll
    for (int l = NI; l < NW; ++l) acc[l] = (uint64_t)accd[l - NI];  // an integer below 2^45: exact
    uint32_t x[NX];
    uint64_t c = 0;
#pragma unroll
    for (int l = 0; l < NW; ++l) {
        const uint64_t t = acc[l] + c;
        x[l] = (uint32_t)t;
        c = t >> 32;
    }
    x[NW] = (uint32_t)c;
    // X = q P + C' with |C'| <= (2^sa + sqrt(k)/2)(2^sb + sqrt(k)/2) < (P / 2)(1 - 2^-20) by the norm rule
    // (sigma_sum_for), so q is the integer nearest X / P, and
    // the estimate from the top three limbs is within 2^-37 of X / P (X < 2^13 P; the dropped
    // limbs are below 2^-37 P): rint gives q exactly, and X - q P is C' itself.
    double xq = 0.0;
#pragma unroll
    for (int l = (NX > 3 ? NX - 3 : 0); l < NX; ++l) xq = fma((double)x[l], cc.kq[l], xq);
    const uint32_t q = (uint32_t)rint(xq);
    uint32_t qp[NX];
    c = 0;
#pragma unroll
    for (int l = 0; l < NX; ++l) {
        const uint64_t t = (uint64_t)q * cc.P[l] + c;
        qp[l] = (uint32_t)t;
        c = t >> 32;
    }
    limbs_addsub<NX, false>(x, qp);  // C', two's complement, |C'| < P / 2
    const bool neg = (int32_t)x[NX - 1] < 0;
    if (neg) {  // magnitude -C'
        uint32_t z[NX];
#pragma unroll
        for (int l = 0; l < NX; ++l) z[l] = 0u;
        limbs_addsub<NX, false>(z, x);
#pragma unroll
        for (int l = 0; l < NX; ++l) x[l] = z[l];
    }
    // The magnitude as 64-bit words; the top nonzero word and the one below it give the
    // leading 64 bits, everything further down only a sticky bit, so the one rounding to 53
    // bits is correct (round to nearest even).
    constexpr int NWD = (NX + 1) / 2;
    uint64_t wd[NWD];
#pragma unroll
    for (int i = 0; i < NWD; ++i)
        wd[i] = (uint64_t)x[2 * i] | (2 * i + 1 < NX ? (uint64_t)x[2 * i + 1] << 32 : 0ull);
    uint64_t hi = wd[0], lo = 0;
    bool sticky = false;
    int ti = 0;
#pragma unroll
    for (int i = 1; i < NWD; ++i) {
        if (wd[i] != 0ull) {
            hi = wd[i];
            lo = wd[i - 1];
            ti = i;
        }
    }
#pragma unroll
    for (int i = 0; i + 2 < NWD; ++i)
        if (i + 2 <= ti && wd[i] != 0ull) sticky = true;
    if (hi == 0ull) return 0.0;
    const int lz = __clzll((long long)hi);
    const uint64_t top64 = lz ? (hi << lz) | (lo >> (64 - lz)) : hi;
    sticky |= (lz ? (lo << lz) : lo) != 0ull;
    const double d = __ull2double_rn(top64 | (uint64_t)sticky);
    const double mag = oz::scale2(d, 64 * ti - lz + shift);
    return neg ? -mag : mag;
    }
}

// Rows row0 .. row0+3 of column col of one product: residue planes [j][col][row] with leading
// dimension res_ld (a multiple of 4).
template <int NW, int NM>
__device__ __forceinline__ void crt_quad(const uint8_t* __restrict__ res, int64_t res_ld, int64_t res_plane,
                                         int64_t m, int64_t row0, int64_t col, const int32_t* __restrict__ row_exp,
                                         const int32_t* __restrict__ col_exp, int ssum, double alpha, double beta_c,
                                         double* __restrict__ C, int64_t ldc, const CrtConst& cc) {
    uint32_t rr[MAX_MODULI];  // four rows' residues per modulus, one byte each
#pragma unroll
    for (int j = 0; j < MAX_MODULI; ++j)
        rr[j] = (NM ? j < NM : j < cc.n) ? *reinterpret_cast<const uint32_t*>(res + j * res_plane + col * res_ld + row0)
                                         : 0u;
    const int f = col_exp[col];
    double* cq = C + row0 + col * ldc;
    if (row0 + 3 < m && (((uintptr_t)cq | (uintptr_t)(row_exp + row0)) & 15) == 0) {
        // a whole quad with 16-byte-aligned exponents and C: one int4 load, two double2 stores
        const int4 e = *reinterpret_cast<const int4*>(row_exp + row0);
        const int ev[4] = {e.x, e.y, e.z, e.w};
        double v[4];
#pragma unroll
        for (int e4 = 0; e4 < 4; ++e4)
            v[e4] = (ev[e4] == oz::EXP_NONFINITE || f == oz::EXP_NONFINITE)
                        ? __longlong_as_double(0x7ff8000000000000ll)
                        : crt_value<NW, NM>(rr, e4, cc, ev[e4] + f - ssum);
        double2* c2 = reinterpret_cast<double2*>(cq);
        double2 lo = make_double2(alpha * v[0], alpha * v[1]), hi = make_double2(alpha * v[2], alpha * v[3]);
        if (beta_c != 0.0) {
            const double2 p0 = c2[0], p1 = c2[1];
            lo = make_double2(fma(alpha, v[0], beta_c * p0.x), fma(alpha, v[1], beta_c * p0.y));
            hi = make_double2(fma(alpha, v[2], beta_c * p1.x), fma(alpha, v[3], beta_c * p1.y));
        }
        c2[0] = lo;
        c2[1] = hi;
        return;
    }
#pragma unroll
    for (int e4 = 0; e4 < 4; ++e4) {
        const int64_t row = row0 + e4;
        if (row >= m) break;
        const int e = row_exp[row];
        double val;
        if (e == oz::EXP_NONFINITE || f == oz::EXP_NONFINITE)
            val = __longlong_as_double(0x7ff8000000000000ll);
        else
            val = crt_value<NW, NM>(rr, e4, cc, e + f - ssum);
        double* cp = C + row + col * ldc;
        *cp = beta_c != 0.0 ? fma(alpha, val, beta_c * *cp) : alpha * val;
    }
}

// The four values of rows row0 .. row0+3 of column col of one product, before alpha (rows at
// or past m: 0).
template <int NW, int NM>
__device__ __forceinline__ void crt_vals(const CrtJob& J, int64_t row0, int64_t col, const CrtConst& cc,
                                         double (&v)[4]) {
    uint32_t rr[MAX_MODULI];
#pragma unroll
    for (int j = 0; j < MAX_MODULI; ++j)
        rr[j] = (NM ? j < NM : j < cc.n)
                    ? *reinterpret_cast<const uint32_t*>(J.res + j * J.res_plane + col * J.res_ld + row0)
                    : 0u;
    const int f = J.col_exp[col];
#pragma unroll
    for (int e4 = 0; e4 < 4; ++e4) {
        v[e4] = 0.0;
        if (row0 + e4 >= J.m) continue;
        const int e = J.row_exp[row0 + e4];
        v[e4] = (e == oz::EXP_NONFINITE || f == oz::EXP_NONFINITE) ? __longlong_as_double(0x7ff8000000000000ll)
                                                                  : crt_value<NW, NM>(rr, e4, cc, e + f - J.bits);
    }
}

// Thread per 4 consecutive rows of one column of C.
template <int NW, int NM>
__global__ void __launch_bounds__(128) crt_reconstruct(const uint8_t* __restrict__ res, int64_t res_ld,
                                                       int64_t res_plane, int64_t m, int64_t n,
                                                       const int32_t* __restrict__ row_exp,
                                                       const int32_t* __restrict__ col_exp, int ssum, double alpha,
                                                       double beta_c, double* __restrict__ C, int64_t ldc,
                                                       const __grid_constant__ CrtConst cc) {
    const int64_t quads = (m + 3) / 4;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= quads * n) return;
    crt_quad<NW, NM>(res, res_ld, res_plane, m, (idx % quads) * 4, idx / quads, row_exp, col_exp, ssum, alpha, beta_c, C,
                 ldc, cc);
}

// Every product of a grouped call: thread -> product by binary search on thread_begin.
template <int NW, int NM>
__global__ void __launch_bounds__(256) crt_grouped(const CrtJob* __restrict__ jobs, int njobs, int64_t threads,
                                                   const __grid_constant__ CrtConst cc) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= threads) return;
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].thread_begin <= idx)
            lo = mid;
        else
            hi = mid - 1;
    }
    const CrtJob& J = jobs[lo];
    const int64_t local = idx - J.thread_begin, quads = (J.m + 3) / 4;
    if (local >= quads * J.n) return;
    const int64_t row0 = (local % quads) * 4, col = local / quads;
    if (J.count <= 1) {
        crt_quad<NW, NM>(J.res, J.res_ld, J.res_plane, J.m, row0, col, J.row_exp, J.col_exp, J.bits, J.alpha, J.beta,
                         J.C, J.ldc, cc);
        return;
    }
    // a stack group: stack 0 as a plain product (alpha v + beta C), then each further stack's
    // alpha v added in stack order -- the stack reduction's order
    double v[4], out[4];
    crt_vals<NW, NM>(J, row0, col, cc, v);
    // (explicitly rounded products and sums: a contracted alpha v + out would skip the rounding
    // of alpha v that the stack-by-stack form makes)
    double* cp = J.C + row0 + col * J.ldc;
#pragma unroll
    for (int e4 = 0; e4 < 4; ++e4)
        out[e4] = (J.beta != 0.0 && row0 + e4 < J.m) ? fma(J.alpha, v[e4], __dmul_rn(J.beta, cp[e4]))
                                                     : __dmul_rn(J.alpha, v[e4]);
    for (int g = 1; g < J.count; ++g) {
        const CrtJob& G = jobs[lo + g];
        crt_vals<NW, NM>(G, row0, col, cc, v);
#pragma unroll
        for (int e4 = 0; e4 < 4; ++e4) out[e4] = __dadd_rn(out[e4], __dmul_rn(G.alpha, v[e4]));
    }
#pragma unroll
    for (int e4 = 0; e4 < 4; ++e4)
        if (row0 + e4 < J.m) cp[e4] = out[e4];
}

cudaError_t launch_qnorm_grouped(cudaStream_t s, const oz::SplitJob* jobs, int njobs, int64_t blocks) {
    qnorm_grouped<<<(unsigned)blocks, 256, 0, s>>>(jobs, njobs);
    return cudaGetLastError();
}

cudaError_t launch_split_residues_grouped(cudaStream_t s, const oz::SplitJob* jobs, int njobs, int64_t blocks,
                                          int nmod, const ModTable& mt) {
    split_residues_grouped<<<(unsigned)blocks, 128, 0, s>>>(jobs, njobs, nmod, mt);
    return cudaGetLastError();
}

cudaError_t launch_crt_grouped(cudaStream_t s, const CrtJob* jobs, int njobs, int64_t threads, const CrtConst& cc,
                               int nmod) {
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    if (nmod == 14)
        crt_grouped<4, 14><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc);
    else if (nmod == 15)
        crt_grouped<4, 15><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc);
    else if (nmod == 16)
        crt_grouped<4, 16><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc);
    else if (nmod == 17)
        crt_grouped<5, 17><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc);
    else if (nmod == 18)
        crt_grouped<5, 18><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc);
    else if (nmod == 19)
        crt_grouped<5, 19><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc);
    else if (nmod == 20)
        crt_grouped<5, 20><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc);
    else
        switch (limbs_for(nmod)) {
            case 2: crt_grouped<2, 0><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc); break;
            case 3: crt_grouped<3, 0><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc); break;
            case 4: crt_grouped<4, 0><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc); break;
            default: crt_grouped<5, 0><<<blocks, 256, 0, s>>>(jobs, njobs, threads, cc); break;
        }
    return cudaGetLastError();
}

}  // namespace oz2

// ---- host orchestration ------------------------------------------------------------------------

template <class CF>
static cudaError_t launch_residue_gemm(const CUtensorMap& tmA, const CUtensorMap& tmB, const oz::Params& prm,
                                       int num_sms, cudaStream_t s) {
    cudaError_t e = smem_opt_in<oz::digit_gemm<CF, 0, 2>>((int)CF::SMEM);
    if (e != cudaSuccess) return e;
    // (tile, modulus) units: as many CTAs (or clusters) as units, up to the SMs
    const int64_t units = (int64_t)prm.tiles_m * prm.tiles_n * prm.ngroups;
    if constexpr (CF::PAIR) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(2 * std::min<int64_t>(units, num_sms / 2)));
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
        return cudaLaunchKernelEx(&cfg, oz::digit_gemm<CF, 0, 2>, tmA, tmB, prm);
    } else {
        oz::digit_gemm<CF, 0, 2><<<(unsigned)std::min<int64_t>(units, num_sms), CF::THREADS, CF::SMEM, s>>>(tmA, tmB,
                                                                                                    prm);
        return cudaGetLastError();
    }
}

static dgt_status ozaki2_dgemm_chunk(dgt_context* h, bool ta, bool tb, int64_t m, int64_t n, int64_t k,
                                     double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
                                     double beta, double* C, int64_t ldc, int nmod);

// K up to KMAX runs as one CRT product; longer K runs as consecutive K-chunks of KMAX, each a
// full CRT product rounded once (beta on the first, accumulation after): one residue product
// must stay exact in INT32, k_pad * 128^2 < 2^31.
dgt_status ozaki2_dgemm(dgt_context* h, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                        const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                        int64_t ldc, int nmod) {
    constexpr int64_t KMAX = 65536;
    if (k <= KMAX) return ozaki2_dgemm_chunk(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, nmod);
    for (int64_t k0 = 0; k0 < k; k0 += KMAX) {
        const int64_t kc = std::min(KMAX, k - k0);
        // op(A) columns k0.. : 'N' -> A + k0 lda, 'T' -> A + k0; op(B) rows k0.. : 'N' -> B + k0, 'T' -> B + k0 ldb
        const double* Ac = ta ? A + k0 : A + k0 * lda;
        const double* Bc = tb ? B + k0 * ldb : B + k0;
        dgt_status st = ozaki2_dgemm_chunk(h, ta, tb, m, n, kc, alpha, Ac, lda, Bc, ldb, k0 == 0 ? beta : 1.0, C,
                                           ldc, nmod);
        if (st != DGT_SUCCESS) return st;
    }
    return DGT_SUCCESS;
}

// Paddings and limits of one CRT product (one K-chunk) with op(B) panels of up to n columns.
dgt_status ozaki2_shape(dgt_context* h, int64_t m, int64_t n, int64_t k, int nmod, Oz2Shape& sh) {
    using namespace oz2;
    if (nmod < MIN_MODULI || nmod > MAX_MODULI)
        return fail(h, DGT_ERROR_INVALID_VALUE, "modulus count must be in [8, 20]");
    const int ssum = sigma_sum_for(nmod, k);
    // kernel variant: 0 (4 epilogue warps), 4 (CTA pair) or 1 (8 warps); all 128-byte stages;
    // 5, 6 and 7 are 1, 4 and 0 with the (tile, modulus) units taken in a dynamic order
    const int ov = h->ozaki_variant;
    const int variant = ov == 5 ? 1 : ov == 6 ? 4 : ov == 7 ? 0 : (ov == 0 || ov == 4) ? ov : 1;
    const bool pair = variant == 4;
    sh.dyn = ov == 5 || ov == 6 || ov == 7;
    const int64_t m_unit = pair ? 2 * oz::TM : oz::TM;
    sh.nmod = nmod;
    sh.sa = (ssum + 1) / 2;
    sh.sb = ssum / 2;
    sh.variant = variant;
    sh.pair = pair;
    sh.m = m;
    sh.k = k;
    sh.m_pad = ceil_div(m, m_unit) * m_unit;
    sh.n_pad = ceil_div(n, oz::TN) * oz::TN;
    sh.k_pad = ceil_div(k, oz::KPAD) * oz::KPAD;
    if (sh.k_pad >= (int64_t)1 << 17)  // k_pad * 128^2 must stay below 2^31
        return fail(h, DGT_ERROR_UNSUPPORTED, "K too long for exact INT32 residue products");
    if ((int64_t)nmod * std::max(sh.m_pad, sh.n_pad) > INT32_MAX)
        return fail(h, DGT_ERROR_UNSUPPORTED, "matrix too large for 32-bit TMA coordinates");
    crt_constants(nmod, sh.cc, sh.mt);
    return DGT_SUCCESS;
}

// amax and residue planes of one operand: the MN rows of op(A) (kcontig = transa) or the MN
// columns of op(B) (kcontig = !transb), planes padded to mn_pad rows.
dgt_status ozaki2_split(dgt_context* h, cudaStream_t s, const Oz2Shape& sh, int sigma, const double* X, int64_t ld,
                        int64_t MN, int64_t mn_pad, bool kcontig, unsigned long long* amax, unsigned long long* qn,
                        int32_t* exps, int8_t* planes, int64_t plane_rows) {
    const int64_t pstride = (plane_rows > 0 ? plane_rows : mn_pad) * sh.k_pad;
    using namespace oz2;
    dgt_status st = ozaki_amax(h, s, X, ld, MN, sh.k, kcontig, amax);
    if (st != DGT_SUCCESS) return st;
    if (kcontig) {
        qnorm_k_contig<<<(unsigned)ceil_div(MN, 8), 256, 0, s>>>(X, ld, MN, sh.k, amax, qn);
    } else {
        DGT_CUDA_TRY(h, cudaMemsetAsync(qn, 0, (size_t)MN * 8, s));
        dim3 g((unsigned)ceil_div(MN, 256), (unsigned)ceil_div(sh.k, oz::AMAX_KCHUNK));
        qnorm_mn_contig<<<g, 256, 0, s>>>(X, ld, MN, sh.k, oz::AMAX_KCHUNK, amax, qn);
    }
    h->launches.fetch_add(1);
    DGT_CUDA_TRY(h, cudaGetLastError());
    dim3 grid((unsigned)ceil_div(mn_pad, RES_ROWS), (unsigned)(sh.k_pad / RES_KSPAN));
    if (kcontig)
        split_residues<true><<<grid, 128, 0, s>>>(X, ld, MN, sh.k, mn_pad, sh.k_pad, pstride, sh.nmod, sigma, amax,
                                                  qn, exps, planes, sh.mt);
    else
        split_residues<false><<<grid, 128, 0, s>>>(X, ld, MN, sh.k, mn_pad, sh.k_pad, pstride, sh.nmod, sigma, amax,
                                                   qn, exps, planes, sh.mt);
    h->launches.fetch_add(1);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DGT_SUCCESS : cuda_fail(h, e, "residue split");
}

// Residue GEMM of split operands (op(A) planes for sh.m rows, op(B) planes for n columns
// padded to n_pad) into res.
// Plane strides: op(A)'s planes a_rows rows apart (0: m_pad), a_span rows addressable from
// planesA (0: nmod a_rows) -- a row panel of a larger operand's planes starts inside them;
// likewise op(B).  The GEMM covers sh.m_pad rows and n_pad columns.
dgt_status ozaki2_residue_gemm(dgt_context* h, cudaStream_t s, const Oz2Shape& sh, int64_t n, int64_t n_pad,
                               const int8_t* planesA, const int8_t* planesB, uint8_t* res, int32_t* sched,
                               int64_t a_rows, int64_t a_span, int64_t b_rows, int64_t b_span) {
    using namespace oz2;
    const int nmod = sh.nmod, tkb = 128;
    const int64_t m = sh.m, m_pad = sh.m_pad, k_pad = sh.k_pad;
    const int64_t m_unit = sh.pair ? 2 * oz::TM : oz::TM;
    const int64_t ars = a_rows > 0 ? a_rows : m_pad, brs = b_rows > 0 ? b_rows : n_pad;
    const int64_t aspan = a_span > 0 ? a_span : (int64_t)nmod * ars, bspan = b_span > 0 ? b_span : (int64_t)nmod * brs;
    if (ars > INT32_MAX || brs > INT32_MAX) return fail(h, DGT_ERROR_UNSUPPORTED, "planes too large");
    CUtensorMap tmA, tmB;
    if (!oz::make_plane_map(&tmA, (void*)planesA, aspan, k_pad, oz::TM, tkb) ||
        !oz::make_plane_map(&tmB, (void*)planesB, bspan, k_pad, sh.pair ? oz::TN / 2 : oz::TN, tkb))
        return fail(h, DGT_ERROR_CUDA, "cuTensorMapEncodeTiled failed");
    static thread_local oz::Params prm;
    prm = oz::Params{};
    prm.m = m;
    prm.n = n;
    prm.ldc = m_pad;
    prm.m_pad = (int32_t)ars;
    prm.n_pad = (int32_t)brs;
    prm.tiles_m = (int32_t)(m_pad / m_unit);
    prm.tiles_n = (int32_t)(n_pad / oz::TN);
    prm.ngroups = nmod;
    for (int j = 0; j < nmod; ++j) {  // one group per modulus: the residue product over all of K
        prm.segs[j] = oz::Seg{j, j, 0, (int32_t)(k_pad / tkb)};
        prm.groups[j] = oz::Group{j, j + 1, 0, sh.mt.p[j]};
    }
    prm.res = res;
    prm.res_ld = m_pad;
    prm.res_plane = m_pad * n_pad;
    prm.err = h->dev_error;
    prm.test_stall = h->test_stall == 1 ? 1 : 0;
    if (sh.dyn && sched) {  // the unit counter starts at zero for every launch
        DGT_CUDA_TRY(h, cudaMemsetAsync(sched, 0, sizeof(int32_t), s));
        prm.sched = sched;
    }
    mark(h, 1);
    cudaError_t le;
    if (sh.variant == 4)
        le = launch_residue_gemm<oz::OzCfg<8, 128, 6, true>>(tmA, tmB, prm, h->num_sms, s);
    else if (sh.variant == 0)
        le = launch_residue_gemm<oz::OzCfg<4, 128, 4>>(tmA, tmB, prm, h->num_sms, s);
    else
        le = launch_residue_gemm<oz::OzCfg<8, 128, 4>>(tmA, tmB, prm, h->num_sms, s);
    h->launches.fetch_add(1);
    if (le != cudaSuccess) return cuda_fail(h, le, "residue GEMM launch");
    return DGT_SUCCESS;
}

// The reconstruction C = alpha C' + beta C of n columns from their residues.
dgt_status ozaki2_reconstruct(dgt_context* h, cudaStream_t s, const Oz2Shape& sh, int64_t n, int64_t n_pad,
                                     const uint8_t* res, const int32_t* expA, const int32_t* expB, double alpha,
                                     double beta, double* C, int64_t ldc) {
    using namespace oz2;
    const int nmod = sh.nmod;
    const int64_t m = sh.m, m_pad = sh.m_pad;
    const int64_t threads = ceil_div(m, 4) * n;
    const unsigned blocks = (unsigned)ceil_div(threads, 128);
    const CrtConst& cc = sh.cc;
    const int bits = sh.sa + sh.sb;
#define DGT_CRT_LAUNCH(NW, NM)                                                                            \
    crt_reconstruct<NW, NM><<<blocks, 128, 0, s>>>(res, m_pad, m_pad * n_pad, m, n, expA, expB, bits, alpha, beta, \
                                                   C, ldc, cc)
    if (nmod == 14)
        DGT_CRT_LAUNCH(4, 14);
    else if (nmod == 15)
        DGT_CRT_LAUNCH(4, 15);
    else if (nmod == 16)
        DGT_CRT_LAUNCH(4, 16);
    else if (nmod == 17)
        DGT_CRT_LAUNCH(5, 17);
    else if (nmod == 18)
        DGT_CRT_LAUNCH(5, 18);
    else if (nmod == 19)
        DGT_CRT_LAUNCH(5, 19);
    else if (nmod == 20)
        DGT_CRT_LAUNCH(5, 20);
    else
        switch (limbs_for(nmod)) {
            case 2: DGT_CRT_LAUNCH(2, 0); break;
            case 3: DGT_CRT_LAUNCH(3, 0); break;
            case 4: DGT_CRT_LAUNCH(4, 0); break;
            default: DGT_CRT_LAUNCH(5, 0); break;
        }
#undef DGT_CRT_LAUNCH
    h->launches.fetch_add(1);
    DGT_CUDA_TRY(h, cudaGetLastError());
    return DGT_SUCCESS;
}

// Residue GEMM and reconstruction of one op(B) panel on one stream.
dgt_status ozaki2_gemm_crt(dgt_context* h, cudaStream_t s, const Oz2Shape& sh, int64_t n, int64_t n_pad,
                           const int8_t* planesA, const int32_t* expA, const int8_t* planesB, const int32_t* expB,
                           uint8_t* res, double alpha, double beta, double* C, int64_t ldc, int32_t* sched) {
    dgt_status st = ozaki2_residue_gemm(h, s, sh, n, n_pad, planesA, planesB, res, sched);
    if (st != DGT_SUCCESS) return st;
    mark(h, 2);
    return ozaki2_reconstruct(h, s, sh, n, n_pad, res, expA, expB, alpha, beta, C, ldc);
}

int64_t ozaki2_n_pad(int64_t n) { return ceil_div(n, oz::TN) * oz::TN; }

// Largest workspace of the CRT scheme for this shape over the kernel variants (the CTA-pair
// variant pads M to 256) and K-chunks (at most 65536 deep); DGT_ERROR_UNSUPPORTED as the call.
dgt_status ozaki2_workspace_bound(int nmod, int64_t m, int64_t n, int64_t k, size_t* bytes) {
    *bytes = 0;
    if (nmod < oz2::MIN_MODULI || nmod > oz2::MAX_MODULI) return DGT_ERROR_INVALID_VALUE;
    const int64_t kc = std::min<int64_t>(std::max<int64_t>(k, 1), 65536);
    for (int pair = 0; pair < 2; ++pair) {
        Oz2Shape sh{};
        sh.nmod = nmod;
        sh.m = m;
        sh.k = kc;
        const int64_t m_unit = pair ? 2 * oz::TM : oz::TM;
        sh.m_pad = ceil_div(m, m_unit) * m_unit;
        sh.n_pad = ceil_div(n, oz::TN) * oz::TN;
        sh.k_pad = ceil_div(kc, oz::KPAD) * oz::KPAD;
        if ((int64_t)nmod * std::max(sh.m_pad, sh.n_pad) > INT32_MAX) return DGT_ERROR_UNSUPPORTED;
        *bytes = std::max(*bytes, ozaki2_carve(sh, n, sh.n_pad, nullptr).bytes);
    }
    return DGT_SUCCESS;
}

// Workspace carve of one CRT product: planes of op(A) (m_pad rows) and op(B) (n_pad rows),
// amax words, exponents and the residue planes of C.
Oz2Work ozaki2_carve(const Oz2Shape& sh, int64_t n, int64_t n_pad, void* ws) {
    auto up = [](size_t x) { return (x + 1023) / 1024 * 1024; };
    const size_t pa = up((size_t)sh.nmod * sh.m_pad * sh.k_pad), pb = up((size_t)sh.nmod * n_pad * sh.k_pad);
    const size_t xa = up((size_t)sh.m * 8), xb = up((size_t)n * 8), ea = up((size_t)sh.m * 4), eb = up((size_t)n * 4);
    const size_t rs = up((size_t)sh.nmod * sh.m_pad * n_pad);
    const size_t sc = 1024;  // the residue GEMM's unit counter (dynamic order)
    Oz2Work w;
    w.bytes = pa + pb + 2 * (xa + xb) + ea + eb + rs + sc;
    char* p = (char*)ws;
    if (!p) return w;
    w.planesA = (int8_t*)p;
    w.planesB = (int8_t*)(p + pa);
    p += pa + pb;
    w.amaxA = (unsigned long long*)p;
    w.amaxB = (unsigned long long*)(p + xa);
    w.qnA = (unsigned long long*)(p + xa + xb);
    w.qnB = (unsigned long long*)(p + 2 * xa + xb);
    p += 2 * (xa + xb);
    w.expA = (int32_t*)p;
    w.expB = (int32_t*)(p + ea);
    w.res = (uint8_t*)(p + ea + eb);
    w.sched = (int32_t*)(p + ea + eb + rs);
    return w;
}

static dgt_status ensure_work_streams(dgt_context* h) {
    for (auto& ws : h->work_stream)
        if (!ws) DGT_CUDA_TRY(h, cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking));
    for (auto& e : h->work_ev)
        if (!e) DGT_CUDA_TRY(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return DGT_SUCCESS;
}

// Panels of op(B) for a device-resident CRT product: the knob's count, else one piece.  (At
// 16384^3, 14 moduli, the CTA-pair kernel: 54.1 ms in one piece, 55.1 ms in 2 or 4 panels,
// 57.1 ms in 8 -- the split and reconstruction blocks that share the SMs slow the residue
// GEMM about as much as they take off the critical path; its 167 registers x 320 threads leave
// room for one 128-thread side block per SM.)
static int crt_panel_count(const dgt_context* h, int64_t, int64_t, int64_t) {
    return h->crt_panels > 0 ? h->crt_panels : 1;
}

// The CRT product with op(B) in np column panels of whole GEMM tiles.  On the handle's
// stream: the split of op(A), then panel by panel the residue GEMM.  On side streams: the
// splits of op(B)'s panels, in order (panel p + 1's while the GEMM runs panel p), and each
// panel's reconstruction once its GEMM is done, while the GEMM runs the next panel.  The
// ALU-bound split and reconstruction kernels so share the SMs with the tensor-bound GEMM
// instead of running before and after it.  Two residue buffers alternate: panel p's GEMM
// waits for panel p - 2's reconstruction.  The side streams fork from and join back into the
// handle's stream through events, so the whole call can be captured in a CUDA graph.  Every
// kernel computes what the one-piece form does for its columns: the results are identical.
static dgt_status ozaki2_dgemm_panels(dgt_context* h, const Oz2Shape& sh, int np, bool ta, bool tb, int64_t n,
                                      double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
                                      double beta, double* C, int64_t ldc) {
    const int64_t pw = ceil_div(ceil_div(n, np), oz::TN) * oz::TN;  // panel width: whole tiles
    np = (int)ceil_div(n, pw);
    auto up = [](size_t x) { return (x + 1023) / 1024 * 1024; };
    const size_t pa = up((size_t)sh.nmod * sh.m_pad * sh.k_pad), pbp = up((size_t)sh.nmod * pw * sh.k_pad);
    const size_t xa = up((size_t)sh.m * 8), xb = up((size_t)n * 8), ea = up((size_t)sh.m * 4), eb = up((size_t)n * 4);
    const size_t rs = up((size_t)sh.nmod * sh.m_pad * pw);
    const size_t bytes = pa + np * pbp + 2 * (xa + xb) + ea + eb + 2 * rs + 1024;
    if (bytes > ozaki2_carve(sh, n, sh.n_pad, nullptr).bytes) return DGT_ERROR_UNSUPPORTED;  // one piece instead
    void* ws = nullptr;
    dgt_status st = ensure_workspace(h, bytes, &ws, 0);
    if (st != DGT_SUCCESS) return st;
    if ((st = ensure_work_streams(h)) != DGT_SUCCESS) return st;
    char* p = (char*)ws;
    int8_t* planesA = (int8_t*)p;
    int8_t* planesB = (int8_t*)(p + pa);
    p += pa + np * pbp;
    auto* amaxA = (unsigned long long*)p;
    auto* amaxB = (unsigned long long*)(p + xa);
    auto* qnA = (unsigned long long*)(p + xa + xb);
    auto* qnB = (unsigned long long*)(p + 2 * xa + xb);
    p += 2 * (xa + xb);
    auto* expA = (int32_t*)p;
    auto* expB = (int32_t*)(p + ea);
    uint8_t* res[2] = {(uint8_t*)(p + ea + eb), (uint8_t*)(p + ea + eb + rs)};
    auto* sched = (int32_t*)(p + ea + eb + 2 * rs);

    cudaStream_t s = h->stream, ss = h->work_stream[0], sr = h->work_stream[1];
    cudaEvent_t* fork = &h->work_ev[0];
    cudaEvent_t* split_done = &h->work_ev[1];
    cudaEvent_t* gemm_done = &h->work_ev[1 + 8];
    cudaEvent_t* recon_done = &h->work_ev[1 + 16];
    mark(h, 0);
    DGT_CUDA_TRY(h, cudaEventRecord(*fork, s));
    DGT_CUDA_TRY(h, cudaStreamWaitEvent(ss, *fork, 0));
    DGT_CUDA_TRY(h, cudaStreamWaitEvent(sr, *fork, 0));
    // op(B)'s panels: 'N' -> columns n0.. at B + n0 ldb (K-contiguous), 'T' -> rows n0.. at B + n0
    for (int q = 0; q < np; ++q) {
        const int64_t n0 = q * pw, w = std::min(pw, n - n0);
        const double* X = tb ? B + n0 : B + n0 * ldb;
        st = ozaki2_split(h, ss, sh, sh.sb, X, ldb, w, pw, !tb, amaxB + n0, qnB + n0, expB + n0,
                          planesB + q * pbp);
        if (st != DGT_SUCCESS) return st;
        DGT_CUDA_TRY(h, cudaEventRecord(split_done[q], ss));
    }
    st = ozaki2_split(h, s, sh, sh.sa, A, lda, sh.m, sh.m_pad, ta, amaxA, qnA, expA, planesA);
    if (st != DGT_SUCCESS) return st;
    for (int q = 0; q < np; ++q) {
        const int64_t n0 = q * pw, w = std::min(pw, n - n0);
        DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, split_done[q], 0));
        if (q >= 2) DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, recon_done[q - 2], 0));
        st = ozaki2_residue_gemm(h, s, sh, w, pw, planesA, planesB + q * pbp, res[q & 1], sched);
        if (st != DGT_SUCCESS) return st;
        DGT_CUDA_TRY(h, cudaEventRecord(gemm_done[q], s));
        DGT_CUDA_TRY(h, cudaStreamWaitEvent(sr, gemm_done[q], 0));
        st = ozaki2_reconstruct(h, sr, sh, w, pw, res[q & 1], expA, expB + n0, alpha, beta, C + n0 * ldc, ldc);
        if (st != DGT_SUCCESS) return st;
        DGT_CUDA_TRY(h, cudaEventRecord(recon_done[q], sr));
    }
    // join: the last reconstruction (every earlier one precedes it on its stream; the splits
    // precede the GEMMs that waited for them)
    DGT_CUDA_TRY(h, cudaStreamWaitEvent(s, recon_done[np - 1], 0));
    mark(h, 2);
    return DGT_SUCCESS;
}

static dgt_status ozaki2_dgemm_chunk(dgt_context* h, bool ta, bool tb, int64_t m, int64_t n, int64_t k,
                                     double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
                                     double beta, double* C, int64_t ldc, int nmod) {
    Oz2Shape sh;
    dgt_status st = ozaki2_shape(h, m, n, k, nmod, sh);
    if (st != DGT_SUCCESS) return st;
    const int np = crt_panel_count(h, m, n, k);
    if (np > 1 && n > oz::TN) {
        // (within the one-piece form's workspace: dgt_dgemm_workspace_size stays a bound)
        st = ozaki2_dgemm_panels(h, sh, std::min(np, 8), ta, tb, n, alpha, A, lda, B, ldb, beta, C, ldc);
        if (st != DGT_ERROR_UNSUPPORTED) return st;
    }
    void* ws = nullptr;
    if ((st = ensure_workspace(h, ozaki2_carve(sh, n, sh.n_pad, nullptr).bytes, &ws, 0)) != DGT_SUCCESS) return st;
    const Oz2Work w = ozaki2_carve(sh, n, sh.n_pad, ws);
    cudaStream_t s = h->stream;
    mark(h, 0);
    // op(A) is m x k: 'N' -> MN-contiguous; op(B) as its transpose n x k: 'N' -> K-contiguous
    if ((st = ozaki2_split(h, s, sh, sh.sa, A, lda, m, sh.m_pad, ta, w.amaxA, w.qnA, w.expA, w.planesA)) !=
        DGT_SUCCESS)
        return st;
    if ((st = ozaki2_split(h, s, sh, sh.sb, B, ldb, n, sh.n_pad, !tb, w.amaxB, w.qnB, w.expB, w.planesB)) !=
        DGT_SUCCESS)
        return st;
    return ozaki2_gemm_crt(h, s, sh, n, sh.n_pad, w.planesA, w.expA, w.planesB, w.expB, w.res, alpha, beta, C, ldc,
                           w.sched);
}

}  // namespace dgt
