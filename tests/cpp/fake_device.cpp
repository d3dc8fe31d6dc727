// Host-memory test double of the CUDA runtime calls and dgt entry points that the 2.5D
// Cannon drivers (include/dgt_drivers.hpp) make, so that their host logic -- allocation
// sizes, copy pitches, the run loop, the result and the CSV rows -- runs and is checked on
// a machine without a GPU (tests/test_csv_log.py links tests/cpp/driver_test.cpp against
// this file instead of libcudart and libdgt).  "Device" memory is host memory, and
// cudaMallocHost marks an allocation page-locked for the *_host entries; kernels are
// plain loops: the Cannon pack / unpack move tile (i, j) <-> &X[lm (j M + i)] with ld M
// (src/25DCannon.cpp:113-136, :254-271) and the multiply computes every C tile as
// alpha sum_t A(i,t) B(t,j) + beta C(i,j), the 2.5D algorithm's result.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <set>
#include <vector>

#include "dgt.h"

struct CUevent_st {
    double t = 0;
};
struct dgt_context {
    int unused = 0;
};

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

extern "C" {

cudaError_t cudaMalloc(void** p, size_t bytes) {
    *p = std::malloc(bytes);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void* p) {
    std::free(p);
    return cudaSuccess;
}
// page-locked allocations, so the *_host entries can tell them from pageable memory
static std::set<const void*> g_pinned;
cudaError_t cudaMallocHost(void** p, size_t bytes) {
    *p = std::malloc(bytes);
    if (!*p) return cudaErrorMemoryAllocation;
    g_pinned.insert(*p);
    return cudaSuccess;
}
cudaError_t cudaFreeHost(void* p) {
    g_pinned.erase(p);
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void* dst, const void* src, size_t bytes, cudaMemcpyKind) {
    std::memcpy(dst, src, bytes);
    return cudaSuccess;
}
cudaError_t cudaMemcpy2D(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                         cudaMemcpyKind) {
    if (width > dpitch || width > spitch) return cudaErrorInvalidPitchValue;
    for (size_t r = 0; r < height; ++r)
        std::memcpy(static_cast<char*>(dst) + r * dpitch, static_cast<const char*>(src) + r * spitch, width);
    return cudaSuccess;
}
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaEventCreate(cudaEvent_t* e) {
    *e = new CUevent_st;
    return cudaSuccess;
}
cudaError_t cudaEventDestroy(cudaEvent_t e) {
    delete e;
    return cudaSuccess;
}
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t) {
    e->t = now_ms();
    return cudaSuccess;
}
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t a, cudaEvent_t b) {
    *ms = float(b->t - a->t);
    return cudaSuccess;
}
const char* cudaGetErrorString(cudaError_t) { return "fake device error"; }

dgt_status dgt_create(dgt_handle_t* h) {
    *h = new dgt_context;
    return DGT_SUCCESS;
}
dgt_status dgt_destroy(dgt_handle_t h) {
    delete h;
    return DGT_SUCCESS;
}
dgt_status dgt_get_stream(dgt_handle_t, dgt_stream_t* s) {
    *s = nullptr;
    return DGT_SUCCESS;
}
dgt_status dgt_check_device(dgt_handle_t) { return DGT_SUCCESS; }
const char* dgt_status_string(dgt_status) { return "fake status"; }
const char* dgt_last_error(dgt_handle_t) { return ""; }

dgt_status dgt_pack_cannon2d(dgt_handle_t, int64_t M, int32_t p, const double* A, const double* B, const double* C,
                             double* const* lA, double* const* lB, double* const* lC) {
    if (p <= 0 || M % p) return DGT_ERROR_INVALID_VALUE;
    const int64_t lm = M / p;
    for (int i = 0; i < p; ++i)
        for (int j = 0; j < p; ++j) {
            const int64_t off = lm * (j * M + i);
            for (int64_t c = 0; c < lm; ++c)
                for (int64_t r = 0; r < lm; ++r) {
                    lA[i * p + j][r + c * lm] = A[off + r + c * M];
                    lB[i * p + j][r + c * lm] = B[off + r + c * M];
                    lC[i * p + j][r + c * lm] = C[off + r + c * M];
                }
        }
    return DGT_SUCCESS;
}

dgt_status dgt_unpack_cannon2d(dgt_handle_t, int64_t M, int32_t p, double* C, const double* const* lC) {
    if (p <= 0 || M % p) return DGT_ERROR_INVALID_VALUE;
    const int64_t lm = M / p;
    for (int i = 0; i < p; ++i)
        for (int j = 0; j < p; ++j)
            for (int64_t c = 0; c < lm; ++c)
                for (int64_t r = 0; r < lm; ++r) C[lm * (j * M + i) + r + c * M] = lC[i * p + j][r + c * lm];
    return DGT_SUCCESS;
}

dgt_status dgt_pack_cannon2d_host(dgt_handle_t h, int64_t M, int32_t p, const double* A, const double* B,
                                  const double* C, double* const* lA, double* const* lB, double* const* lC) {
    if (!g_pinned.count(A) || !g_pinned.count(B) || !g_pinned.count(C)) return DGT_ERROR_INVALID_VALUE;
    return dgt_pack_cannon2d(h, M, p, A, B, C, lA, lB, lC);
}

dgt_status dgt_unpack_cannon2d_host(dgt_handle_t h, int64_t M, int32_t p, double* C, const double* const* lC) {
    if (!g_pinned.count(C)) return DGT_ERROR_INVALID_VALUE;
    return dgt_unpack_cannon2d(h, M, p, C, lC);
}

dgt_status dgt_cannon25d(dgt_handle_t, int64_t M, int32_t p, int32_t c, char ta, char tb, double alpha,
                         const double* const* A, const double* const* B, double beta, double* const* C,
                         dgt_fp64_mode, int) {
    if (p <= 0 || c <= 0 || p % c || M % p) return DGT_ERROR_INVALID_VALUE;
    if ((ta != 'N' && ta != 'n') || (tb != 'N' && tb != 'n')) return DGT_ERROR_UNSUPPORTED;
    const int64_t lm = M / p;
    std::vector<double> acc(size_t(lm * lm));
    for (int i = 0; i < p; ++i)
        for (int j = 0; j < p; ++j) {
            std::fill(acc.begin(), acc.end(), 0.0);
            for (int t = 0; t < p; ++t) {
                const double* a = A[i * p + t];
                const double* b = B[t * p + j];
                for (int64_t col = 0; col < lm; ++col)
                    for (int64_t k = 0; k < lm; ++k) {
                        const double bk = b[k + col * lm];
                        for (int64_t r = 0; r < lm; ++r) acc[r + col * lm] += a[r + k * lm] * bk;
                    }
            }
            double* cc = C[i * p + j];
            for (int64_t e = 0; e < lm * lm; ++e) cc[e] = alpha * acc[e] + beta * cc[e];
        }
    return DGT_SUCCESS;
}

}  // extern "C"
