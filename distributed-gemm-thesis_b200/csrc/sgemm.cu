// FP32 GEMM three ways (the FP32 configuration of the precision study):
//   DGT_FP32_BF16X3: split x = hi + lo with hi = bf16(x), lo = bf16(x - hi); C = alpha *
//                    (lo*hi + hi*lo + hi*hi) + beta*C, all three products accumulated in one
//                    FP32 TMEM accumulator by tcgen05.mma kind::f16 (Henry, Tang, Heinecke 2019)
//   DGT_FP32_BF16X1: the hi*hi product alone
//   DGT_FP32_SIMT:   FP32 FMA on the CUDA cores (register-blocked 128 x 128 tiles)
// The tensor-core modes reuse the digit-GEMM engine (tc_engine.cuh) with BF16 planes and
// its FP32 epilogue.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "dgt_internal.cuh"
#include "tc_engine.cuh"

namespace dgt {
namespace sg {

// FP32 -> BF16 hi/lo planes, K-major [plane][mn_pad][k_pad] (k_pad elements of 2 bytes),
// zero padding.  Each thread produces 32 consecutive k of one mn.
template <bool K_CONTIG>
__global__ void __launch_bounds__(128) split_bf16(const float* __restrict__ X, int64_t ld, int64_t MN, int64_t K,
                                                  int64_t mn_pad, int64_t k_pad, int planes,
                                                  __nv_bfloat16* __restrict__ out) {
    const int64_t mn = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t k0 = (int64_t)blockIdx.y * 32;
    if (mn >= mn_pad) return;
    uint32_t hi[16], lo[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        hi[i] = 0;
        lo[i] = 0;
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const int64_t kk = k0 + i;
        float x = 0.f;
        if (mn < MN && kk < K) x = K_CONTIG ? X[kk + mn * ld] : X[mn + kk * ld];
        __nv_bfloat16 h = __float2bfloat16_rn(x);
        __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
        hi[i >> 1] |= (uint32_t)__bfloat16_as_ushort(h) << (16 * (i & 1));
        lo[i >> 1] |= (uint32_t)__bfloat16_as_ushort(l) << (16 * (i & 1));
    }
    const int64_t plane = mn_pad * k_pad;
    uint4* o = reinterpret_cast<uint4*>(out + mn * k_pad + k0);
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = make_uint4(hi[4 * q], hi[4 * q + 1], hi[4 * q + 2], hi[4 * q + 3]);
    if (planes > 1) {
        uint4* o2 = reinterpret_cast<uint4*>(out + plane + mn * k_pad + k0);
#pragma unroll
        for (int q = 0; q < 4; ++q) o2[q] = make_uint4(lo[4 * q], lo[4 * q + 1], lo[4 * q + 2], lo[4 * q + 3]);
    }
}

// Register-blocked FP32 SIMT GEMM: 128 x 128 tile, 256 threads, 8 x 8 outputs per thread,
// K step 8 through shared memory (A stored k-major, B stored k-major).
constexpr int SB = 128, SK = 8;

__global__ void __launch_bounds__(256) sgemm_simt(int64_t m, int64_t n, int64_t k, float alpha,
                                                  const float* __restrict__ A, int64_t lda, bool ta,
                                                  const float* __restrict__ B, int64_t ldb, bool tb, float beta,
                                                  float* __restrict__ C, int64_t ldc) {
    __shared__ float sA[SK][SB + 4];
    __shared__ float sB[SK][SB + 4];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;  // 16 x 16 threads, 8 x 8 each
    const int64_t m0 = (int64_t)blockIdx.x * SB, n0 = (int64_t)blockIdx.y * SB;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
    for (int64_t k0 = 0; k0 < k; k0 += SK) {
        // 128 x 8 of op(A) and 8 x 128 of op(B): 1024 elements each, 4 per thread
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int e = tid + r * 256;
            const int mm = ta ? (e >> 3) : (e & 127);
            const int kk = ta ? (e & 7) : (e >> 7);
            const int64_t gm = m0 + mm, gk = k0 + kk;
            float va = 0.f;
            if (gm < m && gk < k) va = ta ? A[gk + gm * lda] : A[gm + gk * lda];
            sA[kk][mm] = va;
            const int nn = tb ? (e & 127) : (e >> 3);
            const int kb = tb ? (e >> 7) : (e & 7);
            const int64_t gn = n0 + nn, gkb = k0 + kb;
            float vb = 0.f;
            if (gn < n && gkb < k) vb = tb ? B[gn + gkb * ldb] : B[gkb + gn * ldb];
            sB[kb][nn] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < SK; ++kk) {
            float a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = sA[kk][tx * 4 + (i & 3) + (i >> 2) * 64];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = sB[kk][ty * 4 + (j & 3) + (j >> 2) * 64];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int64_t col = n0 + ty * 4 + (j & 3) + (j >> 2) * 64;
        if (col >= n) continue;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int64_t row = m0 + tx * 4 + (i & 3) + (i >> 2) * 64;
            if (row >= m) continue;
            float* cp = C + row + col * ldc;
            float v = alpha * acc[i][j];
            if (beta != 0.f) v = fmaf(beta, *cp, v);
            *cp = v;
        }
    }
}

}  // namespace sg

static dgt_status sgemm_split(dgt_context* h, bool ta, bool tb, int64_t m, int64_t n, int64_t k, float alpha,
                              const float* A, int64_t lda, const float* B, int64_t ldb, float beta, float* C,
                              int64_t ldc, bool three) {
    const int planes = three ? 2 : 1;
    const int64_t m_pad = ceil_div(m, oz::TM) * oz::TM, n_pad = ceil_div(n, oz::TN) * oz::TN;
    const int64_t k_pad = ceil_div(k, 64) * 64;  // 64 BF16 = one 128-byte stage
    if ((int64_t)planes * std::max(m_pad, n_pad) > INT32_MAX)
        return fail(h, DGT_ERROR_UNSUPPORTED, "matrix too large for 32-bit TMA coordinates");
    std::vector<oz::Seg> segs;
    const int32_t kb = (int32_t)(k_pad / 64);
    if (three) {  // small terms first
        segs.push_back(oz::Seg{1, 0, 0, kb});
        segs.push_back(oz::Seg{0, 1, 0, kb});
    }
    segs.push_back(oz::Seg{0, 0, 0, kb});
    std::vector<oz::Group> groups{oz::Group{0, (int32_t)segs.size(), 0, 0}};
    auto up = [](size_t x) { return (x + 1023) / 1024 * 1024; };
    const size_t pa = up((size_t)planes * m_pad * k_pad * 2), pb = up((size_t)planes * n_pad * k_pad * 2);
    void* ws = nullptr;
    dgt_status st = ensure_workspace(h, pa + pb, &ws, 0);
    if (st != DGT_SUCCESS) return st;
    char* p = (char*)ws;
    __nv_bfloat16* planesA = (__nv_bfloat16*)p;
    __nv_bfloat16* planesB = (__nv_bfloat16*)(p + pa);
    cudaStream_t s = h->stream;
    mark(h, 0);
    {
        dim3 ga((unsigned)(m_pad / 128), (unsigned)(k_pad / 32)), gbd((unsigned)(n_pad / 128), (unsigned)(k_pad / 32));
        // op(A) m x k: 'N' is MN-contiguous; op(B) as n x k: 'N' is K-contiguous
        if (ta)
            sg::split_bf16<true><<<ga, 128, 0, s>>>(A, lda, m, k, m_pad, k_pad, planes, planesA);
        else
            sg::split_bf16<false><<<ga, 128, 0, s>>>(A, lda, m, k, m_pad, k_pad, planes, planesA);
        DGT_LAUNCH_CHECK(h, "split_bf16 A");
        if (!tb)
            sg::split_bf16<true><<<gbd, 128, 0, s>>>(B, ldb, n, k, n_pad, k_pad, planes, planesB);
        else
            sg::split_bf16<false><<<gbd, 128, 0, s>>>(B, ldb, n, k, n_pad, k_pad, planes, planesB);
        DGT_LAUNCH_CHECK(h, "split_bf16 B");
    }
    CUtensorMap tmA, tmB;
    if (!oz::make_plane_map(&tmA, planesA, (int64_t)planes * m_pad, k_pad * 2, oz::TM, 128) ||
        !oz::make_plane_map(&tmB, planesB, (int64_t)planes * n_pad, k_pad * 2, oz::TN, 128))
        return fail(h, DGT_ERROR_CUDA, "cuTensorMapEncodeTiled failed");
    using CF = oz::OzCfg<4, 128, 4>;
    const cudaError_t opt = smem_opt_in<oz::digit_gemm<CF, 1, 1>>((int)CF::SMEM);
    DGT_CUDA_TRY(h, opt);
    static thread_local oz::Params prm;  // ~21 KB: keep it off the stack
    prm = oz::Params{};
    prm.m = m;
    prm.n = n;
    prm.ldc = ldc;
    prm.m_pad = (int32_t)m_pad;
    prm.n_pad = (int32_t)n_pad;
    prm.tiles_m = (int32_t)(m_pad / oz::TM);
    prm.tiles_n = (int32_t)(n_pad / oz::TN);
    prm.ngroups = 1;
    std::copy(segs.begin(), segs.end(), prm.segs);
    std::copy(groups.begin(), groups.end(), prm.groups);
    prm.err = h->dev_error;
    prm.test_stall = h->test_stall == 1 ? 1 : 0;
    prm.Cf = C;
    prm.alpha_f = alpha;
    prm.beta_f = beta;
    const int grid = std::min(prm.tiles_m * prm.tiles_n, h->num_sms);
    mark(h, 1);
    oz::digit_gemm<CF, 1, 1><<<grid, CF::THREADS, CF::SMEM, s>>>(tmA, tmB, prm);
    DGT_LAUNCH_CHECK(h, "digit_gemm bf16");
    mark(h, 2);
    return DGT_SUCCESS;
}

}  // namespace dgt

using namespace dgt;

extern "C" dgt_status dgt_sgemm(dgt_handle_t h, char transa, char transb, int64_t m, int64_t n, int64_t k,
                                const float* alpha, const float* A, int64_t lda, const float* B, int64_t ldb,
                                const float* beta, float* C, int64_t ldc, dgt_fp32_mode mode) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (!alpha || !beta) return fail(h, DGT_ERROR_INVALID_VALUE, "alpha/beta pointer is null");
    if (!valid_op(transa) || !valid_op(transb)) return fail(h, DGT_ERROR_INVALID_VALUE, "transpose must be N, T or C");
    if (m < 0 || n < 0 || k < 0) return fail(h, DGT_ERROR_INVALID_VALUE, "negative dimension");
    const bool ta = is_trans(transa), tb = is_trans(transb);
    if (lda < std::max<int64_t>(1, ta ? k : m)) return fail(h, DGT_ERROR_INVALID_VALUE, "lda < rows of A");
    if (ldb < std::max<int64_t>(1, tb ? n : k)) return fail(h, DGT_ERROR_INVALID_VALUE, "ldb < rows of B");
    if (ldc < std::max<int64_t>(1, m)) return fail(h, DGT_ERROR_INVALID_VALUE, "ldc < m");
    if (m == 0 || n == 0) return DGT_SUCCESS;
    if (!C || (k > 0 && (!A || !B))) return fail(h, DGT_ERROR_INVALID_VALUE, "null matrix pointer");
    if (mode != DGT_FP32_SIMT && mode != DGT_FP32_BF16X1 && mode != DGT_FP32_BF16X3)
        return fail(h, DGT_ERROR_INVALID_VALUE, "unknown FP32 mode");
    if (mode == DGT_FP32_SIMT || k == 0) {
        dim3 grid((unsigned)ceil_div(m, sg::SB), (unsigned)ceil_div(n, sg::SB));
        h->ev_split = false;
        mark(h, 1);
        sg::sgemm_simt<<<grid, 256, 0, h->stream>>>(m, n, k, *alpha, A, lda, ta, B, ldb, tb, *beta, C, ldc);
        DGT_LAUNCH_CHECK(h, "sgemm_simt");
        mark(h, 2);
        return DGT_SUCCESS;
    }
    return sgemm_split(h, ta, tb, m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc, mode == DGT_FP32_BF16X3);
}
