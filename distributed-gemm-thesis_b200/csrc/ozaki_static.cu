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
// device looks up its device address with cudaGetSymbolAddress (with that device current),
// clears the error word and caches both; make that first call before any stream capture
// begins.  Later calls outside a capture look the address up again, so a context that was
// reset (cudaDeviceReset) and recreated is picked up.  Every call on a device shares the
// array and finds the previous call's contents in it: the parts that must start at zero are
// cleared on the stream each time, and calls whose work overlaps on the GPU (two streams,
// or two host threads) race on the scratch.
//
// The error word is sticky: a bounded device wait that ran out in any call sets a bit that
// stays until dgt_ozaki_static_check reads and clears it.
#include <cuda_runtime.h>

#include <mutex>

#include "dgt_internal.cuh"

namespace {

constexpr size_t kErrBytes = 256;  // device error word, padded to keep the planes aligned
__device__ __align__(256) unsigned char g_ozaki_scratch[DGT_OZAKI_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

// With device `dev` current: the array's device address and the SM count.  A device seen for
// the first time (or whose array moved, after a context reset) gets its error word cleared.
// Inside a stream capture only the cached address is used.
dgt_status setup_device(int dev, cudaStream_t s, void** addr, int* sms) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return DGT_ERROR_CUDA;
    if (cs == cudaStreamCaptureStatusNone || !g_scratch_addr[dev]) {
        if (cs != cudaStreamCaptureStatusNone) return DGT_ERROR_NOT_INITIALIZED;  // first call inside a capture
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_ozaki_scratch);
        if (e != cudaSuccess || !p) return DGT_ERROR_CUDA;
        if (p != g_scratch_addr[dev]) {
            int n = 0;
            e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return DGT_ERROR_CUDA;
            if (cudaMemset(p, 0, sizeof(unsigned int)) != cudaSuccess) return DGT_ERROR_CUDA;
            g_num_sms[dev] = n;
            g_scratch_addr[dev] = p;
        }
    }
    *addr = g_scratch_addr[dev];
    *sms = g_num_sms[dev];
    return DGT_SUCCESS;
}

// C = beta C for k = 0 (BLAS: C is not read when beta is 0).
__global__ void scale_c(double* __restrict__ C, int64_t ldc, int64_t m, int64_t n, double beta) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y) {
        double* c = C + i + j * ldc;
        *c = beta == 0.0 ? 0.0 : beta * *c;
    }
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
    size_t need = 0;
    if (k > 0) {
        need = ozaki_scratch_bytes(slices, m, n, k);
        if (need == 0) return DGT_ERROR_UNSUPPORTED;
        // too large for the fixed array: the caller's problem, reported by status alone
        if (need > DGT_OZAKI_STATIC_SCRATCH_BYTES - kErrBytes) return DGT_ERROR_INVALID_VALUE;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DGT_ERROR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    void* base = nullptr;
    int sms = 0;
    dgt_status st = setup_device(dev, s, &base, &sms);
    if (st != DGT_SUCCESS) return st;
    if (k == 0) {  // nothing to multiply: C = beta C
        const dim3 grid((unsigned)((m + 255) / 256), (unsigned)std::min<int64_t>(n, 4096));
        scale_c<<<grid, 256, 0, s>>>(C, ldc, m, n, *beta);
        return cudaGetLastError() == cudaSuccess ? DGT_SUCCESS : DGT_ERROR_CUDA;
    }
    unsigned int* err = (unsigned int*)base;
    return ozaki_dgemm_on(s, sms, err, (char*)base + kErrBytes, DGT_OZAKI_STATIC_SCRATCH_BYTES - kErrBytes, ta, tb,
                          m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc, slices);
}

extern "C" dgt_status dgt_ozaki_static_check(dgt_stream_t stream) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DGT_ERROR_CUDA;
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        base = g_scratch_addr[dev];
    }
    if (!base) return DGT_SUCCESS;  // no call on this device yet: nothing to report
    if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return DGT_ERROR_CUDA;
    unsigned int word = 0;
    if (cudaMemcpy(&word, base, sizeof(word), cudaMemcpyDeviceToHost) != cudaSuccess) return DGT_ERROR_CUDA;
    if (word == 0) return DGT_SUCCESS;
    if (cudaMemset(base, 0, sizeof(word)) != cudaSuccess) return DGT_ERROR_CUDA;
    if (word & DGT_DEVERR_TIMEOUT) return DGT_ERROR_TIMEOUT;
    return DGT_ERROR_INVALID_VALUE;  // a device-side bounds check failed
}
