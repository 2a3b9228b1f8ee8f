// Integer-pipe peak probe: the denominator of the Miller-Rabin roofline.
//
// The squaring engine is bound by 32-bit integer multiplies on the CUDA cores
// (no tensor cores, little DRAM traffic), so its roofline is the device's
// sustained rate of 32-bit multiply instructions.  This kernel runs 8
// independent multiply-add chains per thread on every SM and reports
// multiplies per second, for the low-half form (mul.lo) and the high-half
// form (mul.hi) separately.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace {

constexpr int kIters = 4096;
constexpr int kChains = 8;

__global__ void __launch_bounds__(256) imad_lo_kernel(uint32_t seed, uint32_t *sink) {
    uint32_t a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) a[c] = seed + threadIdx.x * 7u + c;
    const uint32_t k = seed | 1u, d = seed >> 3;
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) a[c] = a[c] * k + d;
    }
    uint32_t r = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) r ^= a[c];
    if (r == 0x9e3779b9u) sink[blockIdx.x] = r;
}

__global__ void __launch_bounds__(256) imad_hi_kernel(uint32_t seed, uint32_t *sink) {
    uint32_t a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) a[c] = seed + threadIdx.x * 7u + c;
    const uint32_t k = seed | 0x80000001u;
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) a[c] = __umulhi(a[c], k) + a[c];
    }
    uint32_t r = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) r ^= a[c];
    if (r == 0x9e3779b9u) sink[blockIdx.x] = r;
}

}  // namespace

// Sustained 32-bit multiply rates of `device` in operations per second.
extern "C" int pfb_measure_int32_peak(int device, double *mul_lo_per_s, double *mul_hi_per_s) {
    PFB_CUDA(cudaSetDevice(device));
    int sms = 0;
    PFB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = sms * 8, threads = 256;
    uint32_t *sink = nullptr;
    PFB_CUDA(cudaMalloc(&sink, sizeof(uint32_t) * blocks));
    cudaEvent_t e0, e1;
    PFB_CUDA(cudaEventCreate(&e0));
    PFB_CUDA(cudaEventCreate(&e1));
    const double ops = (double)blocks * threads * kIters * kChains;
    double best[2] = {0.0, 0.0};
    for (int kind = 0; kind < 2; kind++) {
        for (int rep = 0; rep < 4; rep++) {
            cudaEventRecord(e0);
            if (kind == 0) imad_lo_kernel<<<blocks, threads>>>(0x1234567u + rep, sink);
            else imad_hi_kernel<<<blocks, threads>>>(0x7654321u + rep, sink);
            cudaEventRecord(e1);
            PFB_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            PFB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0 && ms > 0.f) best[kind] = best[kind] > ops / (ms * 1e-3) ? best[kind] : ops / (ms * 1e-3);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (mul_lo_per_s) *mul_lo_per_s = best[0];
    if (mul_hi_per_s) *mul_hi_per_s = best[1];
    return PFB_OK;
}
