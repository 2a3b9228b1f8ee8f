// Shared host/device helpers of the prime-finder B200 engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "pfb_sieve.h"

// A kernel's dynamic shared memory as a 16-byte-aligned array of T.  A macro
// so that a host build of the kernels (the CPU emulation in the tests) can
// supply its own storage.
#ifndef PFB_DYNAMIC_SMEM
#define PFB_DYNAMIC_SMEM(T, name) extern __shared__ __align__(16) T name[]
#endif

namespace pfb {

// Thread-local last-error text behind pfb_last_error().
void set_error(const char *fmt, ...);

// Record a failed CUDA call and return PFB_E_CUDA.
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define PFB_CUDA(expr)                                                        \
    do {                                                                      \
        cudaError_t _e = (expr);                                              \
        if (_e != cudaSuccess) return ::pfb::cuda_fail(_e, #expr, __FILE__, __LINE__); \
    } while (0)

// Modular arithmetic for a 32-bit modulus p >= 2 (Barrett with a 64-bit
// reciprocal m = floor((2^64-1)/p)).  For t < 2^64 the quotient estimate
// umulhi(t, m) is at most 2 below floor(t/p), so two conditional subtractions
// finish the reduction.
struct Mod32 {
    uint32_t p;
    unsigned long long m;

    __device__ __forceinline__ void init(uint32_t p_) {
        p = p_;
        m = ~0ull / (unsigned long long)p_;
    }
    __device__ __forceinline__ uint32_t red(unsigned long long t) const {
        unsigned long long q = __umul64hi(t, m);
        unsigned long long r = t - q * (unsigned long long)p;
        if (r >= p) r -= p;
        if (r >= p) r -= p;
        return (uint32_t)r;
    }
    __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const {
        return red((unsigned long long)a * b);
    }
    // (a - b) mod p for a, b in [0, p); wrap-around of uint32 keeps it exact.
    __device__ __forceinline__ uint32_t sub(uint32_t a, uint32_t b) const {
        uint32_t r = a - b;
        return (a < b) ? r + p : r;
    }
    __device__ __forceinline__ uint32_t pow(uint32_t base, unsigned long long e) const {
        uint32_t r = 1u, x = base;
        while (e) {
            if (e & 1ull) r = mul(r, x);
            x = mul(x, x);
            e >>= 1;
        }
        return r;
    }
};

}  // namespace pfb
