// Pack / unpack kernels: device equivalents of the reference's data decompositions.
//
// Every routine is a permutation of contiguous column runs, so each kernel hands one
// run (a piece of one column that stays contiguous on both sides) to one warp and copies
// it with 16-byte vector loads/stores when both ends allow, 8-byte otherwise.  Runs are
// >= the block size (256-512 doubles at the benchmark shapes), so both the reads and
// the writes are fully coalesced and the kernels are HBM-bound.
//
//  * block-cyclic scatter / gather: pblasDecomposer::scatterMatrix / gatherMatrix
//    (src/Decompositions/pblasDecomposition.cpp:73-221).  Global block (bi, bj) belongs to
//    rank (bi mod p, bj mod q) at local offset ((bi div p)*mb, (bj div q)*nb) -- the
//    closed form of the reference's modular rowOffset/columnOffset walk (:124-130).
//  * strided block batches: copyBlock<double> and copyBlock<float>
//    (src/Transfers/sharedTransfers.cpp:29-63, instantiations :84-88) and the
//    MPI_Type_vector send/recv pairs (src/Transfers/mpiTransfers.cpp:16-57) used by
//    deliverMatrix / gatherResult (2DBlockSequentialDecomposition.cpp:56-253) and
//    decompose2D / reorderMatrix (src/25DCannon.cpp:87-149, :231-284).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "dgt_internal.cuh"

namespace dgt {
namespace {

constexpr int LAYOUT_THREADS = 256;
constexpr int MAX_RANKS = 256;
constexpr int MAX_COPIES = 192;

// Copies n doubles from s to d with one warp (lane = 0..31).  Each lane issues up to four
// 16-byte loads before its stores, so a warp keeps 2 KB in flight per pass.
__device__ __forceinline__ void warp_copy(const double* __restrict__ s, double* __restrict__ d, int64_t n,
                                          int lane) {
    int64_t i = 0;
    if ((((uintptr_t)s ^ (uintptr_t)d) & 15) == 0) {
        // same 16-byte phase: peel one element if needed, then double2
        if (((uintptr_t)s & 15) != 0 && n > 0) {
            if (lane == 0) d[0] = s[0];
            i = 1;
        }
        const double2* s2 = reinterpret_cast<const double2*>(s + i);
        double2* d2 = reinterpret_cast<double2*>(d + i);
        const int64_t pairs = (n - i) >> 1;
        int64_t k = lane;
        for (; k + 96 < pairs; k += 128) {
            double2 v0 = __ldcs(s2 + k), v1 = __ldcs(s2 + k + 32), v2 = __ldcs(s2 + k + 64), v3 = __ldcs(s2 + k + 96);
            __stcs(d2 + k, v0);
            __stcs(d2 + k + 32, v1);
            __stcs(d2 + k + 64, v2);
            __stcs(d2 + k + 96, v3);
        }
        for (; k < pairs; k += 32) __stcs(d2 + k, __ldcs(s2 + k));
        i += pairs * 2;
        if (i < n && lane == 0) d[i] = s[i];
    } else {
        int64_t k = lane;
        for (; k + 96 < n; k += 128) {
            double v0 = __ldcs(s + k), v1 = __ldcs(s + k + 32), v2 = __ldcs(s + k + 64), v3 = __ldcs(s + k + 96);
            __stcs(d + k, v0);
            __stcs(d + k + 32, v1);
            __stcs(d + k + 64, v2);
            __stcs(d + k + 96, v3);
        }
        for (; k < n; k += 32) __stcs(d + k, __ldcs(s + k));
    }
}

// Copies n floats from s to d with one warp: the same scheme with four floats per 16-byte
// vector, so the same-phase case peels up to three head and three tail elements.  Float
// pointers are 4-byte aligned (checked by the caller), so after `head` elements both
// addresses sit on a 16-byte boundary.
__device__ __forceinline__ void warp_copy(const float* __restrict__ s, float* __restrict__ d, int64_t n, int lane) {
    if ((((uintptr_t)s ^ (uintptr_t)d) & 15) == 0) {
        const int64_t head = min(n, (int64_t)(((16 - ((uintptr_t)s & 15)) & 15) >> 2));
        if (lane < head) d[lane] = s[lane];
        const float4* s4 = reinterpret_cast<const float4*>(s + head);
        float4* d4 = reinterpret_cast<float4*>(d + head);
        const int64_t quads = (n - head) >> 2;
        int64_t k = lane;
        for (; k + 96 < quads; k += 128) {
            float4 v0 = __ldcs(s4 + k), v1 = __ldcs(s4 + k + 32), v2 = __ldcs(s4 + k + 64), v3 = __ldcs(s4 + k + 96);
            __stcs(d4 + k, v0);
            __stcs(d4 + k + 32, v1);
            __stcs(d4 + k + 64, v2);
            __stcs(d4 + k + 96, v3);
        }
        for (; k < quads; k += 32) __stcs(d4 + k, __ldcs(s4 + k));
        const int64_t i = head + quads * 4;
        if (lane < n - i) d[i + lane] = s[i + lane];
    } else {
        int64_t k = lane;
        for (; k + 96 < n; k += 128) {
            float v0 = __ldcs(s + k), v1 = __ldcs(s + k + 32), v2 = __ldcs(s + k + 64), v3 = __ldcs(s + k + 96);
            __stcs(d + k, v0);
            __stcs(d + k + 32, v1);
            __stcs(d + k + 64, v2);
            __stcs(d + k + 96, v3);
        }
        for (; k < n; k += 32) __stcs(d + k, __ldcs(s + k));
    }
}

struct CyclicParams {
    int64_t M, N, mb, nb, ldg;
    int32_t p, q;
    int64_t grid_rows;  // ceil(M / mb)
    double* global;
    double* locals[MAX_RANKS];
    int64_t lld[MAX_RANKS];
};

// One run = (global column c, block row bi).
template <bool TO_LOCAL>
__global__ void __launch_bounds__(LAYOUT_THREADS) block_cyclic_kernel(const __grid_constant__ CyclicParams P) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (LAYOUT_THREADS / 32);
    const int64_t runs = P.N * P.grid_rows;
    for (int64_t run = (int64_t)blockIdx.x * (LAYOUT_THREADS / 32) + (threadIdx.x >> 5); run < runs; run += warps) {
        int64_t c = run / P.grid_rows;
        int64_t bi = run - c * P.grid_rows;
        int64_t bj = c / P.nb;
        int rank = (int)(bi % P.p) * P.q + (int)(bj % P.q);
        int64_t lr = (bi / P.p) * P.mb;
        int64_t lc = (bj / P.q) * P.nb + (c - bj * P.nb);
        int64_t r0 = bi * P.mb;
        int64_t len = min(P.mb, P.M - r0);
        double* g = P.global + c * P.ldg + r0;
        double* l = P.locals[rank] + lc * P.lld[rank] + lr;
        if (TO_LOCAL)
            warp_copy(g, l, len, lane);
        else
            warp_copy(l, g, len, lane);
    }
}

template <typename T>
struct CopyDesc {
    const T* src;
    T* dst;
    int64_t ldS, ldD, rows, cols;
    int64_t run_begin;  // prefix sum of cols
};

template <typename T>
struct CopyParams {
    int ncopies;
    int64_t total_runs;
    CopyDesc<T> d[MAX_COPIES];
};

template <typename T>
__global__ void __launch_bounds__(LAYOUT_THREADS) strided_copy_kernel(const __grid_constant__ CopyParams<T> P) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (LAYOUT_THREADS / 32);
    for (int64_t run = (int64_t)blockIdx.x * (LAYOUT_THREADS / 32) + (threadIdx.x >> 5); run < P.total_runs;
         run += warps) {
        int lo = 0, hi = P.ncopies - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (P.d[mid].run_begin <= run)
                lo = mid;
            else
                hi = mid - 1;
        }
        const CopyDesc<T>& cd = P.d[lo];
        int64_t col = run - cd.run_begin;
        warp_copy(cd.src + col * cd.ldS, cd.dst + col * cd.ldD, cd.rows, lane);
    }
}

int layout_grid(dgt_context* h, int64_t runs) {
    int64_t want = ceil_div(runs, LAYOUT_THREADS / 32);
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)h->num_sms * 8));
}

struct ReduceParams {
    int64_t elems;  // per tile
    int tiles, stacks;
    int64_t stack_stride;
    const double* W;
    double* C[MAX_RANKS];
};

// Stack reduction of the 2.5D algorithm: every virtual rank (i,j) adds the partial
// tiles of stacks 1..c-1 into its stack-0 tile (reduceResult, src/25DCannon.cpp:203-228).
__global__ void __launch_bounds__(LAYOUT_THREADS) stack_reduce_kernel(const __grid_constant__ ReduceParams P) {
    const int64_t total = P.elems * P.tiles;
    for (int64_t e = (int64_t)blockIdx.x * LAYOUT_THREADS + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * LAYOUT_THREADS) {
        int t = (int)(e / P.elems);
        int64_t o = e - (int64_t)t * P.elems;
        double v = P.C[t][o];
        for (int s = 0; s < P.stacks; ++s) v += __ldcs(P.W + s * P.stack_stride + e);
        P.C[t][o] = v;
    }
}

struct TileSumParams {
    int64_t elems;
    int nparts;
    double* C;
    const double* parts[MAX_RANKS];
};

// C[e] += parts[0][e] + parts[1][e] + ... in that order (the stack reduction's order), with
// plain loads, so the parts may be other GPUs' memory mapped into this one.
__global__ void __launch_bounds__(LAYOUT_THREADS) tile_sum_kernel(const __grid_constant__ TileSumParams P) {
    for (int64_t e = (int64_t)blockIdx.x * LAYOUT_THREADS + threadIdx.x; e < P.elems;
         e += (int64_t)gridDim.x * LAYOUT_THREADS) {
        double v = P.C[e];
        for (int s = 0; s < P.nparts; ++s) v += P.parts[s][e];
        P.C[e] = v;
    }
}

thread_local CyclicParams t_cyc;
thread_local TileSumParams t_sum;
thread_local CopyParams<double> t_copy;
thread_local CopyParams<float> t_copy_f32;
thread_local ReduceParams t_red;

}  // namespace

dgt_status launch_block_cyclic(dgt_context* h, bool to_local, int64_t M, int64_t N, int64_t mb, int64_t nb, int p,
                               int q, double* global, int64_t ldg, double* const* locals, const int64_t* lld) {
    if (p * q > MAX_RANKS) return fail(h, DGT_ERROR_UNSUPPORTED, "more than 256 virtual ranks");
    CyclicParams& P = t_cyc;
    P.M = M;
    P.N = N;
    P.mb = mb;
    P.nb = nb;
    P.ldg = ldg;
    P.p = p;
    P.q = q;
    P.grid_rows = ceil_div(M, mb);
    P.global = global;
    for (int r = 0; r < p * q; ++r) {
        P.locals[r] = locals[r];
        P.lld[r] = lld[r];
    }
    int64_t runs = N * P.grid_rows;
    if (runs == 0) return DGT_SUCCESS;
    int grid = layout_grid(h, runs);
    if (to_local)
        block_cyclic_kernel<true><<<grid, LAYOUT_THREADS, 0, h->stream>>>(P);
    else
        block_cyclic_kernel<false><<<grid, LAYOUT_THREADS, 0, h->stream>>>(P);
    DGT_LAUNCH_CHECK(h, "block_cyclic_kernel");
    return DGT_SUCCESS;
}

// Strided copies in batches of MAX_COPIES per launch.
dgt_status launch_strided_copies(dgt_context* h, const std::vector<HostCopy>& copies) {
    size_t i = 0;
    while (i < copies.size()) {
        CopyParams<double>& P = t_copy;
        int n = 0;
        int64_t runs = 0;
        for (; i < copies.size() && n < MAX_COPIES; ++i) {
            const HostCopy& c = copies[i];
            if (c.rows <= 0 || c.cols <= 0) continue;
            P.d[n] = CopyDesc<double>{c.src, c.dst, c.ldS, c.ldD, c.rows, c.cols, runs};
            runs += c.cols;
            ++n;
        }
        if (n == 0) continue;
        P.ncopies = n;
        P.total_runs = runs;
        strided_copy_kernel<double><<<layout_grid(h, runs), LAYOUT_THREADS, 0, h->stream>>>(P);
        DGT_LAUNCH_CHECK(h, "strided_copy_kernel");
    }
    return DGT_SUCCESS;
}

// One strided float copy (copyBlock<float>): rows x cols, one warp per column.
dgt_status launch_strided_copy_f32(dgt_context* h, const float* src, float* dst, int64_t ldS, int64_t ldD,
                                   int64_t rows, int64_t cols) {
    if (rows <= 0 || cols <= 0) return DGT_SUCCESS;
    CopyParams<float>& P = t_copy_f32;
    P.ncopies = 1;
    P.total_runs = cols;
    P.d[0] = CopyDesc<float>{src, dst, ldS, ldD, rows, cols, 0};
    strided_copy_kernel<float><<<layout_grid(h, cols), LAYOUT_THREADS, 0, h->stream>>>(P);
    DGT_LAUNCH_CHECK(h, "strided_copy_kernel<float>");
    return DGT_SUCCESS;
}

dgt_status launch_tile_sum(dgt_context* h, double* C, const double* const* parts, int nparts, int64_t elems) {
    if (nparts > MAX_RANKS) return fail(h, DGT_ERROR_UNSUPPORTED, "more than 256 parts");
    TileSumParams& P = t_sum;
    P.elems = elems;
    P.nparts = nparts;
    P.C = C;
    for (int s = 0; s < nparts; ++s) P.parts[s] = parts[s];
    int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(elems, LAYOUT_THREADS), (int64_t)h->num_sms * 8));
    tile_sum_kernel<<<grid, LAYOUT_THREADS, 0, h->stream>>>(P);
    DGT_LAUNCH_CHECK(h, "tile_sum_kernel");
    return DGT_SUCCESS;
}

dgt_status launch_stack_reduce(dgt_context* h, int64_t elems_per_tile, int tiles, int stacks, double* const* C,
                               const double* W, int64_t stack_stride) {
    if (tiles > MAX_RANKS) return fail(h, DGT_ERROR_UNSUPPORTED, "more than 256 tiles");
    ReduceParams& P = t_red;
    P.elems = elems_per_tile;
    P.tiles = tiles;
    P.stacks = stacks;
    P.stack_stride = stack_stride;
    P.W = W;
    for (int t = 0; t < tiles; ++t) P.C[t] = C[t];
    int64_t total = elems_per_tile * tiles;
    int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(total, LAYOUT_THREADS), (int64_t)h->num_sms * 8));
    stack_reduce_kernel<<<grid, LAYOUT_THREADS, 0, h->stream>>>(P);
    DGT_LAUNCH_CHECK(h, "stack_reduce_kernel");
    return DGT_SUCCESS;
}

}  // namespace dgt
