// Device side of the per-operation modular context (pfb_mr_ctx_*, the
// reference's BatchModCtx methods, batch_mod_ctx.cuh:132-179): one CTA per
// modulus runs one operation of the Montgomery engine (mr_device.cuh) on
// operands in the reference's layout -- 16-bit limbs, one per uint64 --
// instead of a whole exponentiation.
//
// Working form ("residue"): x R' mod N, fully reduced (< N), R' = 2^(22 H) + 1
// of the modulus' transform length; the same numbers the engine keeps
// internally in 22-bit limbs, before its final conditional subtraction.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "mr_kernels.cuh"

namespace pfb {
namespace mr {

enum CtxOp : int {
    CTX_MODSQ = 0,    // out = REDC(A^2)         (working form in, working form out)
    CTX_MODMUL = 1,   // out = REDC(A B)
    CTX_RAW_SQ = 2,   // out = A^2, n_sum limbs  (no reduction)
    CTX_RAW_MUL = 3,  // out = A B, n_sum limbs
    CTX_FROM = 4,     // out = A R^-1 mod N      (working form -> plain residue)
};

// Per-modulus buffers beyond the engine's own (JobDev: spectra of N' and N,
// limbs of N, spill buffers of the longest transform).
struct CtxExtra {
    uint32_t *gy;              // [2][L] spectrum of the second factor
    uint32_t *yl;              // H limbs of the second factor
    unsigned long long *raw;   // L coefficients of a raw product
};

// 16-bit limbs (one per uint64, the reference's Data64 layout) -> H limbs of
// 22 bits; limbs past n16 are zero.  dst is padded (shared-memory layout)
// when PAD.
template <bool PAD>
__device__ __forceinline__ void load16(uint32_t *dst, const uint64_t *__restrict__ src, int n16, int H) {
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        const int bit = LIMB_BITS * i, w = bit >> 4, off = bit & 15;
        unsigned long long v = 0;
#pragma unroll
        for (int q = 0; q < 3; q++)
            if (w + q < n16) v |= (unsigned long long)(src[w + q] & 0xFFFFull) << (16 * q);
        dst[PAD ? pad(i) : i] = (uint32_t)(v >> off) & LIMB_MASK;
    }
}

// n16 16-bit limbs (one per uint64) of the value held in H limbs of 22 bits
// at src (padded layout); positions past 22 H bits are zero.
__device__ __forceinline__ void store16(uint64_t *__restrict__ dst, const uint32_t *src, int H, int n16) {
    for (int k = threadIdx.x; k < n16; k += blockDim.x) {
        const int bit = 16 * k, i = bit / LIMB_BITS, off = bit - LIMB_BITS * i;
        unsigned long long v = 0;
        if (i < H) v = src[pad(i)];
        if (i + 1 < H) v |= (unsigned long long)src[pad(i + 1)] << LIMB_BITS;
        dst[k] = (v >> off) & 0xFFFFull;
    }
}

// X <- X - N when X >= N (X < 2N on entry); T: H words of padded scratch.
__device__ __forceinline__ void cond_sub_n(uint32_t *X, uint32_t *T, const uint32_t *__restrict__ nl, int H,
                                           CarrySmem &cs) {
    // X + (B^H - 1 - N) + 1 = X - N + B^H: the carry out is 1 exactly when X >= N
    const unsigned long long c = carry_pass<true>(
        H, 1ull, [&](int i) { return (unsigned long long)X[pad(i)] + (LIMB_MASK - __ldg(nl + i)); }, T, cs);
    if (c)
        for (int i = threadIdx.x; i < H; i += blockDim.x) X[pad(i)] = T[pad(i)];
    __syncthreads();
}

// The full product X Y (gy: the spectrum of Y) or X^2 of the H limbs in
// sm.X, as L limbs of 22 bits in A0 read as one padded array of L words
// (up to L = 2^LOG_LCTA A0 holds them; above, A1 follows A0); no reduction.
// With T(z) = A(z) + z^H C(z) the cyclic product of length H gives c = A + C
// and the negacyclic one d = A - C, coefficient by coefficient, so T's
// coefficients are (c + d) / 2 and (c - d) / 2, both exact; raw holds the 2H
// coefficients between the products and the carry.
template <int LOGL>
__device__ void raw_product_t(const Smem &sm, bool square, const uint32_t *gy, unsigned long long *raw,
                              const Twiddles &tw) {
    constexpr int L = 1 << LOGL, H = L >> 1, LOGH = LOGL - 1;
    const int tid = threadIdx.x;
    uint32_t *A0 = sm.A0, *A1 = sm.A1, *X = sm.X;
    for (int neg = 0; neg < 2; neg++) {
        for (int i = tid; i < H; i += THREADS) {
            const uint32_t v = X[pad(i)];
            A0[pad(i)] = v;
            A1[pad(i)] = v;
        }
        __syncthreads();
        if (!neg) {
            if (square) product_from<true, 0, LOGH, 0, false>(A0, A1, tw, nullptr, nullptr, c_crt);
            else product_from<true, 0, LOGH, 1, true>(A0, A1, tw, gy, gy + L, c_crt);
            for (int i = tid; i < H; i += THREADS) raw[i] = crt(A0[pad(i)], A1[pad(i)], LOGH, c_crt);
        } else {
            if (square) product_from<true, 0, LOGH, 0, false, false, true>(A0, A1, tw, nullptr, nullptr, c_crt);
            else product_from<true, 0, LOGH, 1, true, false, true>(A0, A1, tw, gy + H, gy + L + H, c_crt);
            for (int i = tid; i < H; i += THREADS)  // d as a two's-complement 64-bit value
                raw[H + i] = crt_signed(A0[pad(i)], A1[pad(i)], LOGH, c_crt, 0ull);
        }
        __syncthreads();
    }
    carry_pass<true>(L, 0ull, [&](int i) {
        const int k = i < H ? i : i - H;
        const long long c = (long long)raw[k], d = (long long)raw[H + k];
        return (unsigned long long)((i < H ? c + d : c - d) >> 1);
    }, A0, *sm.cs);
}

__device__ void raw_product(const Smem &sm, int logl, bool square, const uint32_t *gy, unsigned long long *raw,
                            const Twiddles &tw) {
    PFB_LOGL_SWITCH(logl, (raw_product_t<LG>(sm, square, gy, raw, tw)))
}

// One operation on every modulus of a context: CTA b takes modulus b, its
// operands at A + b n16 and B + b n16, its result at out + b out_stride
// (out_stride = n16, or n_sum for the raw products).
__global__ void __launch_bounds__(THREADS, 1)
ctx_kernel(const JobDev *jobs, const CtxExtra *ex, const uint64_t *A, const uint64_t *B, uint64_t *out, int n16,
           int out_stride, int op, Twiddles tw) {
    PFB_DYNAMIC_SMEM(uint32_t, raw);
    const JobDev jb = jobs[blockIdx.x];
    if (jb.phase == 3) return;  // not a valid modulus: nothing to compute
    Smem sm;
    uint32_t *Y;
    carve(raw, jb.logl, sm, Y, jb.ybuf);
    const int L = 1 << jb.logl, H = L >> 1;
    const Cand cd{jb.nn, jb.nh, jb.logl};
    const CtxExtra e = ex[blockIdx.x];
    const size_t b = blockIdx.x;
    uint64_t *o = out + b * (size_t)out_stride;
    load16<true>(sm.X, A + b * (size_t)n16, n16, H);
    if (op == CTX_MODMUL || op == CTX_RAW_MUL) {
        load16<false>(e.yl, B + b * (size_t)n16, n16, H);
        __syncthreads();
        spectrum(sm, jb.logl, e.yl, e.gy, tw);
    }
    __syncthreads();
    switch (op) {
    case CTX_MODSQ:
    case CTX_MODMUL:
        if (op == CTX_MODSQ) mstep(sm, cd, true, 1u, tw, jb);
        else mstep_l(sm, cd, false, 1u, tw, jb, e.gy);
        cond_sub_n(sm.X, sm.A0, jb.nl, H, *sm.cs);
        store16(o, sm.X, H, n16);
        break;
    case CTX_RAW_SQ:
    case CTX_RAW_MUL:
        raw_product(sm, jb.logl, op == CTX_RAW_SQ, e.gy, e.raw, tw);
        __syncthreads();
        store16(o, sm.A0, L, out_stride);
        break;
    case CTX_FROM:
        canonical(sm, Y, cd, jb.nl, tw, jb);
        store16(o, Y, H, n16);
        break;
    }
}

// passed[b] = 1 when the n16 limbs of r equal those of one or of nm1 (the
// working forms of 1 and N - 1), else 0; one CTA per modulus.
__global__ void ctx_check_kernel(const uint64_t *r, const uint64_t *one, const uint64_t *nm1, uint8_t *passed,
                                 int n16) {
    const size_t b = blockIdx.x, o = b * (size_t)n16;
    bool a1 = true, a2 = true;
    for (int k = threadIdx.x; k < n16; k += blockDim.x) {
        const uint64_t v = r[o + k];
        a1 = a1 && (v == one[o + k]);
        a2 = a2 && (v == nm1[o + k]);
    }
    const int m1 = __syncthreads_and(a1), m2 = __syncthreads_and(a2);
    if (threadIdx.x == 0) passed[b] = (uint8_t)(m1 || m2);
}

}  // namespace mr
}  // namespace pfb
