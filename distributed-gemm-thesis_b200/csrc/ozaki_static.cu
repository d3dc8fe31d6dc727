// FP64-accurate GEMM (INT8 Ozaki emulation) that allocates nothing.
//
// Some callers cannot call cudaMalloc at the moment they multiply: processes whose device
// memory is entirely owned by another allocator (a framework's caching pool, a
// pre-reserved arena), and real-time loops that forbid allocation after start-up.  They
// also cannot create a dgt handle, because a handle allocates its error word and grows a
// workspace on demand.  dgt_dgemm_ozaki_static serves them: its scratch (digit planes,
// exponents, the flush schedule and a device error word) lives in one file-scope
// __device__ array of DGT_OZAKI_STATIC_SCRATCH_BYTES that every GPU loading this library
// holds until the process exits.
//
// The array's name is only a host-side stand-in in host code, so the first call on each
// device looks up its device address with cudaGetSymbolAddress (with that device current)
// and caches it; make that first call before any stream capture begins.  Every
// call on a device shares the array and finds the previous call's contents in it: the
// parts that must start at zero are cleared on the stream each time, and calls whose
// work overlaps on the GPU (two streams, or two host threads) race on the scratch.
#include <cuda_runtime.h>

#include <mutex>

#include "dgt_internal.cuh"

#define DGT_OZAKI_STATIC_SCRATCH_BYTES (64ull << 20)

namespace {

constexpr size_t kErrBytes = 256;  // device error word, padded to keep the planes aligned
__device__ __align__(256) unsigned char g_ozaki_scratch[DGT_OZAKI_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

// Once per device, with that device current: the array's device address and SM count.
dgt_status setup_device(int dev, void** addr, int* sms) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_ozaki_scratch);
        if (e != cudaSuccess || !p) return DGT_ERROR_CUDA;
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return DGT_ERROR_CUDA;
        g_num_sms[dev] = n;
        g_scratch_addr[dev] = p;
    }
    *addr = g_scratch_addr[dev];
    *sms = g_num_sms[dev];
    return DGT_SUCCESS;
}

}  // namespace

extern "C" dgt_status dgt_dgemm_ozaki_static(dgt_stream_t stream, char transa, char transb, int64_t m, int64_t n,
                                             int64_t k, const double* alpha, const double* A, int64_t lda,
                                             const double* B, int64_t ldb, const double* beta, double* C,
                                             int64_t ldc, int slices) {
    using namespace dgt;
    if (!alpha || !beta) return DGT_ERROR_INVALID_VALUE;
    if (!valid_op(transa) || !valid_op(transb) || m < 0 || n < 0 || k < 0) return DGT_ERROR_INVALID_VALUE;
    if (slices < 2 || slices > 16) return DGT_ERROR_INVALID_VALUE;
    const bool ta = is_trans(transa), tb = is_trans(transb);
    if (lda < std::max<int64_t>(1, ta ? k : m) || ldb < std::max<int64_t>(1, tb ? n : k) ||
        ldc < std::max<int64_t>(1, m))
        return DGT_ERROR_INVALID_VALUE;
    if (m == 0 || n == 0) return DGT_SUCCESS;
    if (!C || (k > 0 && (!A || !B))) return DGT_ERROR_INVALID_VALUE;
    if (k == 0) return DGT_ERROR_UNSUPPORTED;  // nothing to emulate; use dgt_dgemm
    const size_t need = ozaki_scratch_bytes(slices, m, n, k);
    if (need == 0) return DGT_ERROR_UNSUPPORTED;
    if (need > DGT_OZAKI_STATIC_SCRATCH_BYTES - kErrBytes) {
        std::fprintf(stderr,
                     "dgt_dgemm_ozaki_static: m=%lld n=%lld k=%lld with %d slices needs %zu bytes of scratch; the "
                     "static scratch holds %llu bytes\n",
                     (long long)m, (long long)n, (long long)k, slices, need,
                     (unsigned long long)(DGT_OZAKI_STATIC_SCRATCH_BYTES - kErrBytes));
        return DGT_ERROR_INVALID_VALUE;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DGT_ERROR_CUDA;
    void* base = nullptr;
    int sms = 0;
    dgt_status st = setup_device(dev, &base, &sms);
    if (st != DGT_SUCCESS) return st;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned int* err = (unsigned int*)base;
    if (cudaMemsetAsync(err, 0, sizeof(unsigned int), s) != cudaSuccess) return DGT_ERROR_CUDA;
    return ozaki_dgemm_on(s, sms, err, (char*)base + kErrBytes, DGT_OZAKI_STATIC_SCRATCH_BYTES - kErrBytes, ta, tb,
                          m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc, slices);
}
