// Host test doubles for the CUDA runtime and cuBLAS calls made by the reference's
// hot-path sources (src/Transfers/sharedTransfers.cpp, src/25DCannon.cpp), so they
// run on the CPU inside the oracle.  "Device" memory is host memory from a pool that
// keeps freed blocks mapped (host_pool.h); cudaMemcpy is memcpy; cublasDgemm is a host FP64 GEMM (OpenBLAS when the caller registers its
// cblas_dgemm, else a plain column-major triple loop).  Test infrastructure only.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <sched.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "host_pool.h"
#include "shim_decls.h"

typedef void (*cblas_dgemm_fn)(int order, int ta, int tb, int m, int n, int k, double alpha, const double* A, int lda,
                               const double* B, int ldb, double beta, double* C, int ldc);

// Size-keyed free list of host blocks (host_pool.h).  Blocks are never returned to the
// system; the pool holds at most the peak of one run.
static std::mutex g_pool_mutex;
static std::multimap<size_t, void*> g_pool_free;
static std::unordered_map<void*, size_t> g_pool_size;

void* host_pool_alloc(size_t bytes) {
    const size_t n = (bytes + 63) / 64 * 64;
    {
        std::lock_guard<std::mutex> g(g_pool_mutex);
        auto it = g_pool_free.find(n);
        if (it != g_pool_free.end()) {
            void* p = it->second;
            g_pool_free.erase(it);
            return p;
        }
    }
    void* p = std::aligned_alloc(64, n ? n : 64);
    if (p) {
        std::lock_guard<std::mutex> g(g_pool_mutex);
        g_pool_size[p] = n;
    }
    return p;
}

void host_pool_free(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> g(g_pool_mutex);
    auto it = g_pool_size.find(p);
    if (it == g_pool_size.end()) return;
    g_pool_free.emplace(it->second, p);
}

// Large copies run as one contiguous part per host core (parts of at least 4 MiB); a
// part per core keeps the double's copies near the host's memory bandwidth.
static unsigned host_cores() {
    cpu_set_t set;
    if (sched_getaffinity(0, sizeof(set), &set) == 0) return (unsigned)std::max(1, CPU_COUNT(&set));
    return std::max(1u, std::thread::hardware_concurrency());
}

template <class F>
static void split_parts(size_t bytes, F&& part) {
    const size_t kMinPart = (size_t)4 << 20;
    const size_t parts = std::min<size_t>(host_cores(), bytes / kMinPart);
    if (parts <= 1) {
        part((size_t)0, bytes);
        return;
    }
    const size_t chunk = (bytes / parts + 63) / 64 * 64;
    std::vector<std::thread> ts;
    for (size_t b = chunk; b < bytes; b += chunk) ts.emplace_back([&, b] { part(b, std::min(bytes, b + chunk)); });
    part((size_t)0, std::min(bytes, chunk));
    for (auto& t : ts) t.join();
}

void host_copy(void* dst, const void* src, size_t bytes) {
    char* d = static_cast<char*>(dst);
    const char* s = static_cast<const char*>(src);
    if (d == s || bytes == 0) return;
    if (d < s + bytes && s < d + bytes) {  // overlapping ranges keep memmove's ordering
        std::memmove(d, s, bytes);
        return;
    }
    split_parts(bytes, [&](size_t b, size_t e) { std::memcpy(d + b, s + b, e - b); });
}

void host_zero(void* dst, size_t bytes) {
    char* d = static_cast<char*>(dst);
    split_parts(bytes, [&](size_t b, size_t e) { std::memset(d + b, 0, e - b); });
}

static cblas_dgemm_fn g_host_dgemm = nullptr;
static int g_grid_rows = 1, g_grid_cols = 1;
static long long g_dgemm_calls = 0;
static std::mutex g_calls_mutex;

extern "C" void ref_set_dgemm(void* fn) { g_host_dgemm = (cblas_dgemm_fn)fn; }
extern "C" void* ref_get_dgemm(void) { return (void*)g_host_dgemm; }
extern "C" void ref_set_process_grid(int dRow, int dCol) {
    g_grid_rows = dRow;
    g_grid_cols = dCol;
}
extern "C" long long ref_dgemm_calls(void) { return g_dgemm_calls; }

// Returns the grid the runner asked for (the reference leaves this undefined).
void calculateProcessGrid(int* dRow, int* dCol, int size) {
    (void)size;
    *dRow = g_grid_rows;
    *dCol = g_grid_cols;
}

extern "C" {

cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaGetDevice(int* d) {
    *d = 0;
    return cudaSuccess;
}
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
const char* cudaGetErrorString(cudaError_t) { return "host test double"; }
// Zero-filled, as this double has always handed it out.
cudaError_t cudaMalloc(void** p, size_t n) {
    *p = host_pool_alloc(n ? n : 1);
    if (!*p) return cudaErrorMemoryAllocation;
    host_zero(*p, n ? n : 1);
    return cudaSuccess;
}
cudaError_t cudaFree(void* p) {
    host_pool_free(p);
    return cudaSuccess;
}
cudaError_t cudaMemGetInfo(size_t* free_b, size_t* total_b) {
    *free_b = (size_t)1 << 40;
    *total_b = (size_t)1 << 40;
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void* dst, const void* src, size_t count, enum cudaMemcpyKind) {
    host_copy(dst, src, count);
    return cudaSuccess;
}
cudaError_t cudaMemcpy2D(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                         enum cudaMemcpyKind) {
    for (size_t r = 0; r < height; ++r)
        std::memmove((char*)dst + r * dpitch, (const char*)src + r * spitch, width);
    return cudaSuccess;
}
cudaError_t cudaPointerGetAttributes(struct cudaPointerAttributes* a, const void*) {
    std::memset(a, 0, sizeof(*a));
    a->type = cudaMemoryTypeHost;
    return cudaSuccess;
}

cublasStatus_t cublasCreate_v2(cublasHandle_t* h) {
    *h = (cublasHandle_t)std::malloc(16);
    return CUBLAS_STATUS_SUCCESS;
}
cublasStatus_t cublasDestroy_v2(cublasHandle_t h) {
    std::free((void*)h);
    return CUBLAS_STATUS_SUCCESS;
}

cublasStatus_t cublasDgemm_v2(cublasHandle_t, cublasOperation_t transa, cublasOperation_t transb, int m, int n, int k,
                              const double* alpha, const double* A, int lda, const double* B, int ldb,
                              const double* beta, double* C, int ldc) {
    {
        std::lock_guard<std::mutex> g(g_calls_mutex);
        ++g_dgemm_calls;
    }
    bool ta = transa != CUBLAS_OP_N, tb = transb != CUBLAS_OP_N;
    if (g_host_dgemm) {
        g_host_dgemm(102, ta ? 112 : 111, tb ? 112 : 111, m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc);
        return CUBLAS_STATUS_SUCCESS;
    }
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < m; ++i) {
            double s = 0.0;
            for (int p = 0; p < k; ++p) {
                double a = ta ? A[p + (long long)i * lda] : A[i + (long long)p * lda];
                double b = tb ? B[j + (long long)p * ldb] : B[p + (long long)j * ldb];
                s += a * b;
            }
            double& c = C[i + (long long)j * ldc];
            c = (*beta == 0.0) ? (*alpha) * s : (*alpha) * s + (*beta) * c;
        }
    }
    return CUBLAS_STATUS_SUCCESS;
}

}  // extern "C"

// Used only by the reference's benchmark drivers (src/25DCannon.cpp:392-538), which the
// oracle does not call; defined so that the translation unit links.
template <typename T>
void MatrixInit(T* matrix, const long long size, int) {
    for (long long i = 0; i < size; ++i) matrix[i] = 0;
}
template void MatrixInit<double>(double*, const long long, int);
