// Peak-rate probes: register-resident loops with no memory traffic, timed with CUDA
// events on the handle's stream.  They give the measured FP64 ceilings that the native
// GEMM's roofline fraction is reported against (DMMA = FP64 tensor pipe, DFMA = FP64
// CUDA cores).
#include <cuda_runtime.h>

#include "dgt_internal.cuh"

namespace dgt {
namespace {

constexpr int PROBE_THREADS = 256;
constexpr int PROBE_ITERS = 4096;

__global__ void __launch_bounds__(PROBE_THREADS) dmma_probe_kernel(double* out, double seed) {
    double acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[i][e] = 0.0;
    double a0 = seed + threadIdx.x * 1e-9, a1 = seed * 0.5, b0 = seed * 0.25;
    for (int it = 0; it < PROBE_ITERS; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            asm volatile(
                "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                : "+d"(acc[i][0]), "+d"(acc[i][1]), "+d"(acc[i][2]), "+d"(acc[i][3])
                : "d"(a0), "d"(a1), "d"(b0));
        }
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += acc[i][0] + acc[i][1] + acc[i][2] + acc[i][3];
    if (s == 12345.678) out[0] = s;  // keeps the loop live; never true for the probe inputs
}

// The same with the m16n8k16 shape (4x the FLOPs per instruction).
__global__ void __launch_bounds__(PROBE_THREADS) dmma16_probe_kernel(double* out, double seed) {
    double acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[i][e] = 0.0;
    const double a = seed + threadIdx.x * 1e-9, b = seed * 0.25;
    for (int it = 0; it < PROBE_ITERS / 4; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            asm volatile(
                "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%4,%4,%4,%4,%4,%4,%4}, "
                "{%5,%5,%5,%5}, {%0,%1,%2,%3};\n"
                : "+d"(acc[i][0]), "+d"(acc[i][1]), "+d"(acc[i][2]), "+d"(acc[i][3])
                : "d"(a), "d"(b));
        }
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += acc[i][0] + acc[i][1] + acc[i][2] + acc[i][3];
    if (s == 12345.678) out[0] = s;
}

__global__ void __launch_bounds__(PROBE_THREADS) dfma_probe_kernel(double* out, double seed) {
    double acc[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i] = seed * i;
    const double a = 1.0000001, b = 1e-9 * threadIdx.x;
    for (int it = 0; it < PROBE_ITERS; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i] = fma(acc[i], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += acc[i];
    if (s == 12345.678) out[0] = s;
}

// Half the warps of each block run the DMMA loop, half the DFMA loop: shows whether the
// FP64 tensor pipe and the FP64 FMA pipe run concurrently.
__global__ void __launch_bounds__(PROBE_THREADS) mixed_probe_kernel(double* out, double seed) {
    if ((threadIdx.x >> 5) & 1) {
        double acc[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i] = seed * i;
        const double a = 1.0000001, b = 1e-9 * threadIdx.x;
        for (int it = 0; it < PROBE_ITERS * 16; ++it) {  // same FLOPs as a DMMA warp
#pragma unroll
            for (int i = 0; i < 8; ++i) acc[i] = fma(acc[i], a, b);
        }
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) s += acc[i];
        if (s == 12345.678) out[0] = s;
    } else {
        double acc[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][e] = 0.0;
        double a0 = seed + threadIdx.x * 1e-9, a1 = seed * 0.5, b0 = seed * 0.25;
        for (int it = 0; it < PROBE_ITERS; ++it) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                asm volatile(
                    "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                    : "+d"(acc[i][0]), "+d"(acc[i][1]), "+d"(acc[i][2]), "+d"(acc[i][3])
                    : "d"(a0), "d"(a1), "d"(b0));
            }
        }
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) s += acc[i][0] + acc[i][1] + acc[i][2] + acc[i][3];
        if (s == 12345.678) out[0] = s;
    }
}

}  // namespace
}  // namespace dgt

using namespace dgt;

extern "C" dgt_status dgt_probe_peak(dgt_handle_t h, int32_t kind, double* tflops) {
    if (!h) return DGT_ERROR_NOT_INITIALIZED;
    if (!tflops || kind < 0 || kind > 3) return fail(h, DGT_ERROR_INVALID_VALUE, "bad probe kind");
    void* ws = nullptr;
    dgt_status st = ensure_workspace(h, 64, &ws, 1);
    if (st != DGT_SUCCESS) return st;
    const int blocks = h->num_sms * 4;
    cudaEvent_t e0, e1;
    DGT_CUDA_TRY(h, cudaEventCreate(&e0));
    DGT_CUDA_TRY(h, cudaEventCreate(&e1));
    float best_ms = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {  // first run is warm-up
        cudaEventRecord(e0, h->stream);
        if (kind == 0)
            dmma_probe_kernel<<<blocks, PROBE_THREADS, 0, h->stream>>>((double*)ws, 1.0);
        else if (kind == 1)
            dfma_probe_kernel<<<blocks, PROBE_THREADS, 0, h->stream>>>((double*)ws, 1.0);
        else if (kind == 3)
            dmma16_probe_kernel<<<blocks, PROBE_THREADS, 0, h->stream>>>((double*)ws, 1.0);
        else
            mixed_probe_kernel<<<blocks, PROBE_THREADS, 0, h->stream>>>((double*)ws, 1.0);
        h->launches.fetch_add(1);
        cudaEventRecord(e1, h->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) return cuda_fail(h, e, "probe");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best_ms) best_ms = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double warps = (double)blocks * PROBE_THREADS / 32.0;
    double flops;
    if (kind == 0 || kind == 3)
        flops = warps * PROBE_ITERS * 8 * (2.0 * 16 * 8 * 4);  // per warp-level m16n8k4 (k16: a quarter as many)
    else if (kind == 1)
        flops = (double)blocks * PROBE_THREADS * PROBE_ITERS * 8 * 2.0;
    else  // half the warps each, equal FLOPs per warp
        flops = warps / 2 * PROBE_ITERS * 8 * (2.0 * 16 * 8 * 4) + (warps / 2) * 32 * PROBE_ITERS * 16 * 8 * 2.0;
    *tflops = flops / (best_ms * 1e-3) / 1e12;
    return DGT_SUCCESS;
}
