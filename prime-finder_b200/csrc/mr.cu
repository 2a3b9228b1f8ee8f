// Batched Miller-Rabin engine: kernels and host driver.
//
// One CTA per candidate runs its whole chain of Montgomery squarings on chip
// (mr_device.cuh).  The host side does the per-modulus set-up the reference
// does with GMP (barrett.cu:58-107, montgomery.cu:30-45,
// miller_rabin_runner.cu:315-325): N' = -N^-1 mod R, R mod N, N - 1 = 2^s d.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "bigint_host.h"
#include "common.cuh"
#include "lucas_host.h"
#include "mr_device.cuh"
#include "mr_tables_host.h"
#include "pfb_mr.h"

namespace pfb {
namespace mr {

__constant__ CrtConsts c_crt;

// State of one candidate in device memory.
struct JobDev {
    uint32_t *x;          // H limbs: Montgomery residue (working value)
    uint32_t *res;        // H limbs: canonical residue a^E mod N (output)
    uint32_t *nph;        // [2][L] NTT_L(N')
    uint32_t *nh;         // [2][H] NTT_H(N)
    const uint32_t *npl;  // H limbs of N' (set-up input)
    const uint32_t *nl;   // H limbs of N
    const uint32_t *exp;  // exponent, 32-bit words, little-endian
    uint32_t *spill_s;    // L words  (sequential-prime step only)
    uint32_t *spill_t;    // H words  (sequential-prime step only)
    uint32_t *ybuf;       // H words  (sequential-prime step only: canonical residue)
    struct LucasDev *lucas;  // strong Lucas test (mode 2) only
    int logl;
    int cursor;   // next exponent bit (MSB first); phase 0 while >= 0
    int extra;    // squarings left in phase 2 (s - 1 for a strong test)
    int phase;    // 0 exponent loop, 1 first check, 2 squarings r < s, 3 done
    uint32_t base;
    int mode;     // 0 modular power only, 1 strong test, 2 strong Lucas test
    int verdict;  // 1 probable prime, 0 composite
    int steps;    // steps taken (diagnostics)
};

// Strong Lucas state of one candidate: H limbs each, Montgomery form: V_k,
// V_(k+1), Q^k, a product, R mod N; gy the [2][L] spectrum of V_(k+1).
struct LucasDev {
    uint32_t *lv0, *lv1, *lqk, *lt, *lone, *gy;
    int q;        // Selfridge Q = (1 - D) / 4
    uint32_t lb;  // every stored value is < lb * N
};

// Shared memory: both primes' transforms + X + Y up to L = 2^LOG_LCTA; one
// transform + X above (the sequential-prime step keeps Y in global memory).
__host__ __device__ inline size_t smem_words(int logl) {
    const size_t L = (size_t)1 << logl, H = L / 2;
    return logl <= LOG_LCTA ? 2 * (L + L / 32) + 2 * (H + H / 32) : (L + L / 32) + (H + H / 32);
}
inline size_t smem_bytes(int logl) {
    return smem_words(logl) * sizeof(uint32_t) + sizeof(CarrySmem) + 16;
}

__device__ __forceinline__ void carve(uint32_t *raw, int logl, Smem &sm, uint32_t *&Y, uint32_t *ybuf) {
    const int L = 1 << logl, H = L >> 1;
    sm.A0 = raw;
    if (logl <= LOG_LCTA) {
        sm.A1 = raw + L + L / 32;
        sm.X = sm.A1 + L + L / 32;
        Y = sm.X + H + H / 32;
    } else {
        sm.A1 = nullptr;
        sm.X = raw + L + L / 32;
        Y = ybuf;
    }
    uintptr_t c = (uintptr_t)(raw + smem_words(logl));
    c = (c + 15) & ~(uintptr_t)15;
    sm.cs = (CarrySmem *)c;
}

__global__ void __launch_bounds__(THREADS, 1) prep_kernel(JobDev *jobs, const int *list, Twiddles tw) {
    extern __shared__ __align__(16) uint32_t raw[];
    const JobDev jb = jobs[list ? list[blockIdx.x] : (int)blockIdx.x];
    if (jb.phase == 3) return;
    Smem sm;
    uint32_t *Y;
    carve(raw, jb.logl, sm, Y, jb.ybuf);
    const int L = 1 << jb.logl, H = L >> 1;
    if (jb.logl <= LOG_LCTA) {
        for (int i = threadIdx.x; i < L; i += blockDim.x) {
            const uint32_t v = i < H ? jb.npl[i] : 0u;
            sm.A0[pad(i)] = v;
            sm.A1[pad(i)] = v;
        }
        __syncthreads();
        dif(sm.A0, sm.A1, jb.logl, tw);
        for (int i = threadIdx.x; i < L; i += blockDim.x) {
            jb.nph[i] = red2(sm.A0[pad(i)], P1);
            jb.nph[L + i] = red2(sm.A1[pad(i)], P2);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < H; i += blockDim.x) {
            sm.A0[pad(i)] = jb.nl[i];
            sm.A1[pad(i)] = jb.nl[i];
        }
        __syncthreads();
        dif(sm.A0, sm.A1, jb.logl - 1, tw);
        for (int i = threadIdx.x; i < H; i += blockDim.x) {
            jb.nh[i] = red2(sm.A0[pad(i)], P1);
            jb.nh[H + i] = red2(sm.A1[pad(i)], P2);
        }
        return;
    }
    uint32_t *A = sm.A0;
    for (int pr = 0; pr < 2; pr++) {
        for (int i = threadIdx.x; i < L; i += blockDim.x) A[pad(i)] = i < H ? jb.npl[i] : 0u;
        __syncthreads();
        if (pr == 0) dif1<0>(A, jb.logl, tw);
        else dif1<1>(A, jb.logl, tw);
        const uint32_t p = pr ? P2 : P1;
        for (int i = threadIdx.x; i < L; i += blockDim.x) jb.nph[pr * L + i] = red2(A[pad(i)], p);
        __syncthreads();
        for (int i = threadIdx.x; i < H; i += blockDim.x) A[pad(i)] = jb.nl[i];
        __syncthreads();
        if (pr == 0) dif1<0>(A, jb.logl - 1, tw);
        else dif1<1>(A, jb.logl - 1, tw);
        for (int i = threadIdx.x; i < H; i += blockDim.x) jb.nh[pr * H + i] = red2(A[pad(i)], p);
        __syncthreads();
    }
}

// One Montgomery step in the layout chosen by the transform length (gy: the
// spectrum of a second factor, see mont_step).
template <bool MUL>
__device__ __forceinline__ void mstep_t(const Smem &sm, const Cand &cd, bool square, uint32_t a, const Twiddles &tw,
                                        const JobDev &jb, const uint32_t *gy) {
    static_assert(LOG_LCTA == 14 && LOG_LSEQ == 15, "length cases below");
    switch (cd.logl) {
#define PFB_STEP(n)                                                  \
    case n:                                                          \
        mont_step<MUL, n>(sm, cd, square, a, tw, c_crt, gy);        \
        break;
        PFB_STEP(8) PFB_STEP(9) PFB_STEP(10) PFB_STEP(11) PFB_STEP(12) PFB_STEP(13) PFB_STEP(14)
#undef PFB_STEP
    default: {
        const Spill sp{jb.spill_s, jb.spill_t};
        mont_step_seq<MUL, LOG_LSEQ>(sm, cd, square, a, tw, c_crt, sp, gy);
    }
    }
}

// The strong test's squarings (inlined into its loop).
__device__ __forceinline__ void mstep(const Smem &sm, const Cand &cd, bool square, uint32_t a, const Twiddles &tw,
                                      const JobDev &jb) {
    mstep_t<false>(sm, cd, square, a, tw, jb, nullptr);
}

// The Lucas ladder's steps: one out-of-line copy with the general product, so
// the strong test's loop keeps its own register allocation.
__device__ __noinline__ void mstep_l(const Smem &sm, const Cand &cd, bool square, uint32_t a, const Twiddles &tw,
                                     const JobDev &jb, const uint32_t *gy) {
    mstep_t<true>(sm, cd, square, a, tw, jb, gy);
}

// Canonical residue of X (Montgomery form) into Y: Y = X R^-1 mod N.
template <bool LUCAS = false>
__device__ void canonical(const Smem &sm, uint32_t *Y, const Cand &cd, const uint32_t *nl, const Twiddles &tw,
                          const JobDev &jb) {
    const int H = 1 << (cd.logl - 1);
    for (int i = threadIdx.x; i < H; i += blockDim.x) Y[pad(i)] = sm.X[pad(i)];
    __syncthreads();
    Smem s2 = sm;
    s2.X = Y;
    if (LUCAS) mstep_l(s2, cd, false, 1u, tw, jb, nullptr);
    else mstep(s2, cd, false, 1u, tw, jb);
    // REDC(X) lies in [0, N]; it is N only when X == 0 (mod N), e.g. a base
    // that is a multiple of N.  Map it to 0.
    bool eqn = true;
    for (int i = threadIdx.x; i < H; i += blockDim.x) eqn = eqn && (Y[pad(i)] == nl[i]);
    if (__syncthreads_and(eqn))
        for (int i = threadIdx.x; i < H; i += blockDim.x) Y[pad(i)] = 0u;
    __syncthreads();
}

// ------------------------------------------------------- strong Lucas ----
// Selfridge's method A (P = 1, Q = (1 - D)/4) on the squaring engine.  With
// N + 1 = 2^s d, d odd, N is a strong Lucas probable prime when U_d == 0 or
// V_(d 2^r) == 0 (mod N) for some 0 <= r < s.  The ladder keeps (V_k,
// V_(k+1), Q^k) and for each bit b of d, from the top, moves k to 2k + b:
//   V_2k = V_k^2 - 2 Q^k,  V_2k+1 = V_k V_(k+1) - Q^k,  V_2k+2 = V_(k+1)^2 - 2 Q^(k+1),
// Q^2k = (Q^k)^2, Q^(2k+1) = Q (Q^k)^2.  Since D U_k = 2 V_(k+1) - V_k and
// gcd(D, N) = 1, U_d == 0 is tested as V_d - 2 V_(d+1) == 0.
// Values are kept below lb N (lb = 2 + 4 Q^2) and R > lb^2 N keeps every
// product's REDC below 2N.

__device__ __forceinline__ void load_res(uint32_t *X, const uint32_t *src, int H) {
    for (int i = threadIdx.x; i < H; i += blockDim.x) X[pad(i)] = __ldcg(src + i);
    __syncthreads();
}

__device__ __forceinline__ void store_res(uint32_t *dst, const uint32_t *X, int H) {
    for (int i = threadIdx.x; i < H; i += blockDim.x) dst[i] = X[pad(i)];
    __syncthreads();
}

// g[2][L] <- NTT_L of the H limbs at src (zero-padded), both primes, reduced.
__device__ void spectrum(const Smem &sm, int logl, const uint32_t *src, uint32_t *g, const Twiddles &tw) {
    const int L = 1 << logl, H = L >> 1;
    if (logl <= LOG_LCTA) {
        for (int i = threadIdx.x; i < L; i += blockDim.x) {
            const uint32_t v = i < H ? __ldcg(src + i) : 0u;
            sm.A0[pad(i)] = v;
            sm.A1[pad(i)] = v;
        }
        __syncthreads();
        dif(sm.A0, sm.A1, logl, tw);
        for (int i = threadIdx.x; i < L; i += blockDim.x) {
            g[i] = red2(sm.A0[pad(i)], P1);
            g[L + i] = red2(sm.A1[pad(i)], P2);
        }
        __syncthreads();
        return;
    }
    uint32_t *A = sm.A0;
    for (int pr = 0; pr < 2; pr++) {
        for (int i = threadIdx.x; i < L; i += blockDim.x) A[pad(i)] = i < H ? __ldcg(src + i) : 0u;
        __syncthreads();
        if (pr == 0) dif1<0>(A, logl, tw);
        else dif1<1>(A, logl, tw);
        const uint32_t p = pr ? P2 : P1;
        for (int i = threadIdx.x; i < L; i += blockDim.x) g[pr * L + i] = red2(A[pad(i)], p);
        __syncthreads();
    }
}

// out <- x + c y (sub = false) or x + c (m N - y) (sub = true: x - c y mod N,
// for y < m N), over H limbs; x(i) and y(i) read limb i of the operands
// (x may return 0).  m N - y is formed as m N + (B^H - 1 - y) + 1 - B^H so
// every coefficient is non-negative; the B^H term is the carry out of the
// top limb, dropped (the result itself is below R = B^H).
template <bool OPAD, class GX, class GY>
__device__ void lincomb(uint32_t *out, GX x, GY y, const uint32_t *nl, uint32_t c, uint32_t m, bool sub, int H,
                        CarrySmem &cs) {
    const unsigned long long cm = (unsigned long long)c * m;
    if (sub)
        carry_pass<OPAD>(H, 0ull, [&](int i) {
            return x(i) + cm * __ldg(nl + i) + (unsigned long long)c * (LIMB_MASK - y(i)) + (i == 0 ? c : 0u);
        }, out, cs);
    else
        carry_pass<OPAD>(H, 0ull, [&](int i) { return x(i) + (unsigned long long)c * y(i); }, out, cs);
}

// Is the value in X zero mod N?  (Y receives its canonical residue.)
__device__ bool residue_zero(const Smem &sm, uint32_t *Y, const Cand &cd, const JobDev &jb, const Twiddles &tw) {
    canonical<true>(sm, Y, cd, jb.nl, tw, jb);
    const int H = 1 << (cd.logl - 1);
    bool z = true;
    for (int i = threadIdx.x; i < H; i += blockDim.x) z = z && (Y[pad(i)] == 0u);
    return __syncthreads_and(z) != 0;
}

// One ladder bit: (V_k, V_(k+1), Q^k) -> k' = 2k + bit.
__device__ void lucas_bit(const Smem &sm, const Cand &cd, const JobDev &jb, const LucasDev &lc, uint32_t bit,
                          const Twiddles &tw) {
    const int H = 1 << (cd.logl - 1);
    CarrySmem &cs = *sm.cs;
    const uint32_t aq = (uint32_t)(lc.q < 0 ? -lc.q : lc.q), mq = 2u * aq;  // Q^k < 2|Q| N
    uint32_t *X = sm.X;
    auto gX = [&](int i) { return (unsigned long long)X[pad(i)]; };
    auto g0 = [&](int) { return 0ull; };
    auto glt = [&](int i) { return (unsigned long long)__ldcg(lc.lt + i); };
    auto gqk = [&](int i) { return (unsigned long long)__ldcg(lc.lqk + i); };
    // T1 = V_k V_(k+1) -> lt
    spectrum(sm, cd.logl, lc.lv1, lc.gy, tw);
    load_res(X, lc.lv0, H);
    mstep_l(sm, cd, false, 1u, tw, jb, lc.gy);
    store_res(lc.lt, X, H);
    // T2 = V_k^2 (bit 0) or V_(k+1)^2 (bit 1), in X
    load_res(X, bit ? lc.lv1 : lc.lv0, H);
    mstep_l(sm, cd, true, 1u, tw, jb, nullptr);
    if (!bit) {
        lincomb<false>(lc.lv0, gX, gqk, jb.nl, 2u, mq, true, H, cs);   // V_2k   = T2 - 2 Q^k
        lincomb<false>(lc.lv1, glt, gqk, jb.nl, 1u, mq, true, H, cs);  // V_2k+1 = T1 - Q^k
    } else {
        lincomb<false>(lc.lv0, glt, gqk, jb.nl, 1u, mq, true, H, cs);  // V_2k+1 = T1 - Q^k
        // V_2k+2 = T2 - 2 Q Q^k
        lincomb<false>(lc.lv1, gX, gqk, jb.nl, 2u * aq, mq, lc.q > 0, H, cs);
    }
    if (aq == 1u) {  // Q = -1: Q^k' = (-1)^k' = (-1)^bit
        auto gone = [&](int i) { return (unsigned long long)__ldcg(lc.lone + i); };
        lincomb<false>(lc.lqk, g0, gone, jb.nl, 1u, 2u, bit != 0u, H, cs);
    } else {
        load_res(X, lc.lqk, H);
        mstep_l(sm, cd, true, bit ? aq : 1u, tw, jb, nullptr);  // (Q^k)^2 |Q|^bit < 2 |Q| N
        lincomb<false>(lc.lqk, g0, gX, jb.nl, 1u, mq, bit && lc.q < 0, H, cs);
    }
}

// Strong Lucas steps of one candidate (mode 2); returns steps taken.
__device__ __noinline__ int run_lucas(JobDev &jb, const Smem &sm, uint32_t *Y, int max_steps, const Twiddles &tw, int &cursor,
                         int &phase, int &extra, int &verdict) {
    const Cand cd{jb.nph, jb.nh, jb.logl};
    const LucasDev lc = *jb.lucas;
    const int H = 1 << (jb.logl - 1);
    CarrySmem &cs = *sm.cs;
    const uint32_t aq = (uint32_t)(lc.q < 0 ? -lc.q : lc.q), mq = 2u * aq;
    auto g0 = [&](int) { return 0ull; };
    auto gqk = [&](int i) { return (unsigned long long)__ldcg(lc.lqk + i); };
    auto gX = [&](int i) { return (unsigned long long)sm.X[pad(i)]; };
    int steps = 0;
    while (steps < max_steps && phase != 3) {
        if (phase == 0) {
            const uint32_t bit = (__ldg(jb.exp + (cursor >> 5)) >> (cursor & 31)) & 1u;
            lucas_bit(sm, cd, jb, lc, bit, tw);
            cursor--;
            if (cursor < 0) phase = 1;
        } else {
            if (phase == 2) {  // V_2m = V_m^2 - 2 Q^m, Q^2m = (Q^m)^2
                load_res(sm.X, lc.lv0, H);
                mstep_l(sm, cd, true, 1u, tw, jb, nullptr);
                lincomb<false>(lc.lv0, gX, gqk, jb.nl, 2u, mq, true, H, cs);
                if (aq == 1u) {  // Q^2m = 1
                    auto gone = [&](int i) { return (unsigned long long)__ldcg(lc.lone + i); };
                    lincomb<false>(lc.lqk, g0, gone, jb.nl, 1u, 2u, false, H, cs);
                } else {
                    load_res(sm.X, lc.lqk, H);
                    mstep_l(sm, cd, true, 1u, tw, jb, nullptr);
                    store_res(lc.lqk, sm.X, H);
                }
                extra--;
            }
            bool hit = false;
            if (phase == 1) {  // U_d == 0  <=>  V_d - 2 V_(d+1) == 0
                auto gv0 = [&](int i) { return (unsigned long long)__ldcg(lc.lv0 + i); };
                auto gv1 = [&](int i) { return (unsigned long long)__ldcg(lc.lv1 + i); };
                lincomb<true>(sm.X, gv0, gv1, jb.nl, 2u, lc.lb, true, H, cs);
                hit = residue_zero(sm, Y, cd, jb, tw);
            }
            if (!hit) {  // V_(d 2^r) == 0
                load_res(sm.X, lc.lv0, H);
                hit = residue_zero(sm, Y, cd, jb, tw);
            }
            if (hit) {
                verdict = 1;
                phase = 3;
            } else if (extra <= 0) {
                verdict = 0;
                phase = 3;
            } else {
                phase = 2;
            }
        }
        steps++;
    }
    return steps;
}

// Runs up to max_steps steps of one candidate.  The job's state is read with
// L2 loads (__ldcg): in the persistent kernel another SM may have written it
// earlier in the same launch.
__device__ void run_job(JobDev *jp, int max_steps, const Twiddles &tw, uint32_t *raw) {
    JobDev jb;
    {
        const unsigned long long *src = reinterpret_cast<const unsigned long long *>(jp);
        unsigned long long *dst = reinterpret_cast<unsigned long long *>(&jb);
#pragma unroll
        for (int w = 0; w < (int)(sizeof(JobDev) / 8); w++) dst[w] = __ldcg(src + w);
    }
    if (jb.phase == 3) return;
    Smem sm;
    uint32_t *Y;
    carve(raw, jb.logl, sm, Y, jb.ybuf);
    const int H = 1 << (jb.logl - 1);
    const Cand cd{jb.nph, jb.nh, jb.logl};
    int cursor = jb.cursor, phase = jb.phase, extra = jb.extra, verdict = jb.verdict, steps = 0;
    if (jb.mode == 2) {
        steps = run_lucas(jb, sm, Y, max_steps, tw, cursor, phase, extra, verdict);
        if (threadIdx.x == 0) {
            jp->cursor = cursor;
            jp->phase = phase;
            jp->extra = extra;
            jp->verdict = verdict;
            jp->steps = jb.steps + steps;
        }
        __syncthreads();
        return;
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) sm.X[pad(i)] = __ldcg(jb.x + i);
    __syncthreads();

    while (steps < max_steps && phase != 3) {
        if (phase == 0) {
            const uint32_t bit = (__ldg(jb.exp + (cursor >> 5)) >> (cursor & 31)) & 1u;
            mstep(sm, cd, true, bit ? jb.base : 1u, tw, jb);
            cursor--;
            if (cursor < 0) phase = 1;
        } else {
            if (phase == 2) {
                mstep(sm, cd, true, 1u, tw, jb);
                extra--;
            }
            canonical(sm, Y, cd, jb.nl, tw, jb);
            // compare with 1 and N - 1 (N odd: N - 1 differs from N in limb 0 only)
            bool one = true, nm1 = true;
            for (int i = threadIdx.x; i < H; i += blockDim.x) {
                const uint32_t y = Y[pad(i)], nli = jb.nl[i];
                one = one && (y == (i == 0 ? 1u : 0u));
                nm1 = nm1 && (y == (i == 0 ? nli - 1u : nli));
            }
            const int all_one = __syncthreads_and(one);
            const int all_nm1 = __syncthreads_and(nm1);
            if (phase == 1)
                for (int i = threadIdx.x; i < H; i += blockDim.x) jb.res[i] = Y[pad(i)];
            if (jb.mode == 0) {
                phase = 3;
            } else if (all_nm1 || (phase == 1 && all_one)) {
                verdict = 1;
                phase = 3;
            } else if (extra <= 0) {
                verdict = 0;
                phase = 3;
            } else {
                phase = 2;
            }
        }
        steps++;
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) jb.x[i] = sm.X[pad(i)];
    if (threadIdx.x == 0) {
        jp->cursor = cursor;
        jp->phase = phase;
        jp->extra = extra;
        jp->verdict = verdict;
        jp->steps = jb.steps + steps;
    }
    __syncthreads();
}

// Persistent scheduler: one CTA per SM takes quanta (`quantum` steps of one
// candidate) until `total` quanta are handed out.  Quantum q goes to the
// first unfinished, unlocked candidate at or after q mod n, so candidates
// advance round-robin and no SM idles while work remains.  Nothing waits: a
// CTA that finds every candidate locked or finished leaves.
__global__ void __launch_bounds__(THREADS, 1)
persist_kernel(JobDev *jobs, int n, int *locks, unsigned int *counter, unsigned int total, int quantum,
               Twiddles tw) {
    extern __shared__ __align__(16) uint32_t raw[];
    __shared__ int s_job;
    for (;;) {
        if (threadIdx.x == 0) {
            int job = -1;
            const unsigned int q = atomicAdd(counter, 1u);
            if (q < total) {
                for (int probe = 0; probe < n; probe++) {
                    const int j = (int)((q + (unsigned int)probe) % (unsigned int)n);
                    if (__ldcg(&jobs[j].phase) == 3) continue;
                    if (atomicCAS(&locks[j], 0, 1) != 0) continue;
                    __threadfence();
                    if (__ldcg(&jobs[j].phase) != 3) {
                        job = j;
                        break;
                    }
                    atomicExch(&locks[j], 0);
                }
            }
            s_job = job;
        }
        __syncthreads();
        const int j = s_job;
        __syncthreads();
        if (j < 0) break;
        run_job(jobs + j, quantum, tw, raw);
        if (threadIdx.x == 0) {
            __threadfence();
            atomicExch(&locks[j], 0);
        }
    }
}

// ---------------------------------------------------------------- host ----


struct HostPrep {
    int ok = 0;        // 1 = valid
    int decided = -1;  // >= 0: verdict known without device work (Lucas: a factor, a square)
    int logl = 0;
    int s = 0;
    std::vector<uint32_t> x0, npl, nl, exp;
    int cursor = 0;
    int n16 = 0;  // limbs of N (16-bit)
    int q = 0;                 // Lucas: Q
    uint32_t lb = 0;           // Lucas: value bound factor
    std::vector<uint32_t> v0;  // Lucas: V_0 = 2 in Montgomery form
};

static int choose_logl(size_t nbits, uint32_t base) {
    const int abits = 32 - __builtin_clz(base);
    for (int lg = LOG_LMIN; lg <= LOG_LSEQ; lg++) {
        const size_t rbits = (size_t)LIMB_BITS << (lg - 1);
        if (rbits >= nbits + 2 + 2 * (size_t)abits) return lg;
    }
    return -1;
}

// mode 1: exponent d of N - 1 = 2^s d; mode 0: exponent given; mode 2: the
// strong Lucas test, exponent d of N + 1 = 2^s d.
static void host_prep(const pfb_mr_number_t &num, uint32_t base, int mode, const pfb_mr_number_t *ex,
                      HostPrep &hp) {
    using namespace pfb::big;
    hp.ok = 0;
    if (!num.limbs || num.n_limbs <= 0) return;
    Words N = from_u16(num.limbs, (size_t)num.n_limbs);
    const size_t nb = bit_length(N);
    if (nb < 2 || !(N[0] & 1ull) || nb > (size_t)PFB_MR_MAX_BITS) return;
    if (mode == 2) {
        long D = 0;
        const int sel = selfridge(N, D);
        if (sel < 0) return;
        if (sel == 0) {
            hp.ok = 1;
            hp.decided = 0;
            return;
        }
        hp.q = (int)((1 - D) / 4);
        const uint32_t aq = (uint32_t)(hp.q < 0 ? -hp.q : hp.q);
        hp.lb = 2u + 4u * aq * aq;
        base = hp.lb;
    }
    const int lg = choose_logl(nb, base);
    if (lg < 0) return;
    const size_t H = (size_t)1 << (lg - 1);
    const size_t rbits = LIMB_BITS * H;
    Words E;
    int s = 0;
    if (mode == 1) {
        Words nm1 = sub_small(N, 1);
        while (!test_bit(nm1, (size_t)s)) s++;
        E = shr(nm1, (size_t)s);
    } else if (mode == 2) {
        Words np1 = N;
        size_t i = 0;
        while (i < np1.size() && ++np1[i] == 0) i++;
        if (i == np1.size()) np1.push_back(1);
        while (!test_bit(np1, (size_t)s)) s++;
        E = shr(np1, (size_t)s);
    } else {
        if (!ex || !ex->limbs || ex->n_limbs <= 0) return;
        E = from_u16(ex->limbs, (size_t)ex->n_limbs);
        if (E.empty()) return;
    }
    hp.logl = lg;
    hp.s = s;
    hp.n16 = num.n_limbs;
    hp.npl.assign(H, 0);
    hp.nl.assign(H, 0);
    hp.x0.assign(H, 0);
    to_limbs(neg_inv_pow2(N, rbits), LIMB_BITS, hp.npl.data(), H);
    to_limbs(N, LIMB_BITS, hp.nl.data(), H);
    const Words x0 = pow2_mod(rbits, N);
    to_limbs(x0, LIMB_BITS, hp.x0.data(), H);
    if (mode == 2) {
        hp.v0.assign(H, 0);
        to_limbs(mul_small(x0, 2), LIMB_BITS, hp.v0.data(), H);
    }
    const size_t eb = bit_length(E);
    hp.cursor = (int)eb - 1;
    hp.exp.assign((eb + 31) / 32 + 1, 0);
    for (size_t i = 0; i < eb; i++)
        if (test_bit(E, i)) hp.exp[i / 32] |= 1u << (i % 32);
    hp.ok = 1;
}

}  // namespace mr
}  // namespace pfb

using namespace pfb::mr;

struct pfb_mr {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    uint32_t *d_tw = nullptr;
    uint32_t *d_wide = nullptr;
    Twiddles tw{};
    // persistent-kernel parameters per transform length (pfb_mr_autotune):
    // steps of one candidate per quantum, steps per launch
    int quantum[LOG_LMAX + 1];
    int chunk[LOG_LMAX + 1];
};

static int build_tables(pfb_mr *e) {
    const int half = 1 << (LOG_LMAX - 1);
    const std::vector<uint32_t> h = twiddle_table();
    PFB_CUDA(cudaMalloc(&e->d_tw, h.size() * sizeof(uint32_t)));
    PFB_CUDA(cudaMemcpy(e->d_tw, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    for (int pr = 0; pr < 2; pr++) {
        uint32_t *base = e->d_tw + (size_t)(4 * pr) * half;
        e->tw.w[pr] = base;
        e->tw.wsh[pr] = base + half;
        e->tw.wi[pr] = base + 2 * half;
        e->tw.wish[pr] = base + 3 * half;
    }
    const CrtConsts cc = crt_consts();
    PFB_CUDA(cudaMemcpyToSymbol(c_crt, &cc, sizeof(cc)));
    WideTabs wt{};
    const std::vector<uint32_t> wide = wide_tables(h, wt);
    PFB_CUDA(cudaMalloc(&e->d_wide, wide.size() * sizeof(uint32_t)));
    PFB_CUDA(cudaMemcpy(e->d_wide, wide.data(), wide.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    wt.base = (const uint4 *)e->d_wide;
    PFB_CUDA(cudaMemcpyToSymbol(c_wide, &wt, sizeof(wt)));
    return PFB_OK;
}

extern "C" int pfb_mr_device(const pfb_mr_t *e) { return e ? e->device : -1; }

extern "C" int pfb_mr_create(pfb_mr_t **out, int device) {
    if (!out) {
        pfb::set_error("pfb_mr_create: null out");
        return PFB_E_ARG;
    }
    *out = nullptr;
    pfb_mr *e = new pfb_mr();
    e->device = device;
    for (int lg = 0; lg <= LOG_LMAX; lg++) {
        e->quantum[lg] = 64;
        e->chunk[lg] = 2048;
    }
    int rc = PFB_OK;
    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "cudaSetDevice", __FILE__, __LINE__);
    if (!rc) {
        ce = cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, device);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "attr", __FILE__, __LINE__);
    }
    if (!rc) {
        ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "stream", __FILE__, __LINE__);
    }
    if (!rc) rc = build_tables(e);
    if (!rc) {
        const int mx = (int)std::max(smem_bytes(LOG_LCTA), smem_bytes(LOG_LSEQ));
        ce = cudaFuncSetAttribute(persist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        if (ce == cudaSuccess) ce = cudaFuncSetAttribute(prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "smem attribute", __FILE__, __LINE__);
    }
    if (rc) {
        if (e->stream) cudaStreamDestroy(e->stream);
        cudaFree(e->d_tw);
        delete e;
        return rc;
    }
    *out = e;
    return PFB_OK;
}

extern "C" void pfb_mr_destroy(pfb_mr_t *e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) {
        cudaStreamSynchronize(e->stream);
        cudaStreamDestroy(e->stream);
    }
    cudaFree(e->d_tw);
    cudaFree(e->d_wide);
    delete e;
}

namespace {

// Per-candidate device layout inside the arena (32-bit words).
struct Layout {
    size_t x, res, nph, nh, npl, nl, exp, ss, st, yb, lv0, lv1, lqk, lt, lone, gy, total;
};

Layout layout_for(int logl, size_t exp_words, bool lucas = false) {
    const size_t L = (size_t)1 << logl, H = L / 2;
    Layout l{};
    size_t o = 0;
    auto take = [&](size_t words) {
        const size_t at = o;
        o += (words + 63) & ~(size_t)63;  // 256-byte alignment
        return at;
    };
    l.x = take(H);
    l.res = take(H);
    l.nph = take(2 * L);
    l.nh = take(2 * H);
    l.npl = take(H);
    l.nl = take(H);
    l.exp = take(exp_words);
    if (logl > LOG_LCTA) {
        l.ss = take(L);
        l.st = take(H);
        l.yb = take(H + H / 32);  // padded like the shared-memory residue
    }
    if (lucas) {
        l.lv0 = take(H);
        l.lv1 = take(H);
        l.lqk = take(H);
        l.lt = take(H);
        l.lone = take(H);
        l.gy = take(2 * L);
    }
    l.total = o;
    return l;
}

Layout layout_for(const HostPrep &hp, bool lucas) { return layout_for(hp.logl, hp.exp.size(), lucas); }

// Slot layout of the server: the exponent region sized for the longest
// modulus of the length class, so that slots of one class are interchangeable.
Layout slot_layout(int logl) {
    const size_t H = (size_t)1 << (logl - 1);
    return layout_for(logl, (LIMB_BITS * H + 31) / 32 + 1);
}

void prep_all(const pfb_mr_number_t *nums, int n, uint32_t base, int mode, const pfb_mr_number_t *exps,
              std::vector<HostPrep> &hp) {
    hp.resize(n);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::min<unsigned>(hw, (unsigned)std::max(1, n));
    if (nt <= 1 || n < 4) {
        for (int i = 0; i < n; i++) host_prep(nums[i], base, mode, exps ? exps + i : nullptr, hp[i]);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&, t]() {
            for (int i = t; i < n; i += nt) host_prep(nums[i], base, mode, exps ? exps + i : nullptr, hp[i]);
        });
    for (auto &x : th) x.join();
}

}  // namespace

// A set of candidates resident in device memory, advanced step by step.
struct pfb_mr_batch {
    pfb_mr *e = nullptr;
    int n = 0, mode = 1, maxlog = LOG_LMIN, n_ok = 0;
    long long max_steps = 0, steps_done = 0;
    uint8_t *d_arena = nullptr;
    JobDev *d_jobs = nullptr;
    int *d_locks = nullptr;           // [n] per-candidate locks of the persistent kernel
    unsigned int *d_counter = nullptr;  // quanta handed out in the current launch
    LucasDev *d_lucas = nullptr;        // [n] (strong Lucas batches only)
    std::vector<HostPrep> hp;
    std::vector<JobDev> jobs;
    std::vector<LucasDev> lucas;
    struct Graph {
        long long chunk;
        int quantum;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;  // one launch of the persistent kernel per (chunk, quantum)
};

namespace {

void batch_free(pfb_mr_batch *b) {
    for (auto &g : b->graphs) cudaGraphExecDestroy(g.exec);
    cudaFree(b->d_arena);
    delete b;
}

// One step chunk of a batch -- the quanta counter reset and the persistent
// kernel -- as a CUDA graph, built on first use per (chunk, quantum) and
// replayed by every later advance of the batch.
int chunk_graph(pfb_mr_batch *b, long long chunk, int quantum, cudaGraphExec_t *out) {
    for (const auto &g : b->graphs)
        if (g.chunk == chunk && g.quantum == quantum) {
            *out = g.exec;
            return PFB_OK;
        }
    JobDev *jobs = b->d_jobs;
    int n = b->n, q = quantum;
    int *locks = b->d_locks;
    unsigned int *counter = b->d_counter;
    const long long qpj = (chunk + quantum - 1) / quantum;
    unsigned int total = (unsigned int)std::min<long long>((long long)b->n * qpj, 0x7fffffffll);
    Twiddles tw = b->e->tw;
    void *args[] = {&jobs, &n, &locks, &counter, &total, &q, &tw};
    cudaGraph_t graph = nullptr;
    PFB_CUDA(cudaGraphCreate(&graph, 0));
    cudaMemsetParams mp{};
    mp.dst = counter;
    mp.value = 0;
    mp.elementSize = sizeof(unsigned int);
    mp.width = 1;
    mp.height = 1;
    cudaKernelNodeParams kp{};
    kp.func = (void *)persist_kernel;
    kp.gridDim = dim3((unsigned)std::min(b->n, std::max(1, b->e->num_sms)));
    kp.blockDim = dim3(THREADS);
    kp.sharedMemBytes = (unsigned)smem_bytes(b->maxlog);
    kp.kernelParams = args;
    cudaGraphNode_t n_mem = nullptr, n_ker = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t ce = cudaGraphAddMemsetNode(&n_mem, graph, nullptr, 0, &mp);
    if (ce == cudaSuccess) ce = cudaGraphAddKernelNode(&n_ker, graph, &n_mem, 1, &kp);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return pfb::cuda_fail(ce, "chunk graph", __FILE__, __LINE__);
    b->graphs.push_back(pfb_mr_batch::Graph{chunk, quantum, exec});
    *out = exec;
    return PFB_OK;
}

int batch_build(pfb_mr *e, const pfb_mr_number_t *nums, int n, uint32_t base, int mode,
                const pfb_mr_number_t *exps, pfb_mr_batch **out) {
    *out = nullptr;
    if (!e || !nums || n <= 0 || base < 2 || base > 0xFFFFu) {
        pfb::set_error("pfb_mr: bad argument (n=%d base=%u)", n, base);
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(e->device));
    pfb_mr_batch *b = new pfb_mr_batch();
    b->e = e;
    b->n = n;
    b->mode = mode;
    prep_all(nums, n, base, mode, exps, b->hp);
    std::vector<Layout> lay(n);
    size_t total = 0;
    for (int i = 0; i < n; i++) {
        if (!b->hp[i].ok || b->hp[i].decided >= 0) continue;
        lay[i] = layout_for(b->hp[i], mode == 2);
        total += lay[i].total;
        b->maxlog = std::max(b->maxlog, b->hp[i].logl);
        b->max_steps = std::max(b->max_steps, (long long)b->hp[i].cursor + 2 + b->hp[i].s);
        b->n_ok++;
    }
    const size_t job_bytes = ((size_t)n * sizeof(JobDev) + 255) & ~(size_t)255;
    const size_t lock_bytes = ((size_t)n * sizeof(int) + 256 + 255) & ~(size_t)255;
    const size_t lucas_bytes = mode == 2 ? (((size_t)n * sizeof(LucasDev) + 255) & ~(size_t)255) : 0;
    const size_t need = job_bytes + lock_bytes + lucas_bytes + total * sizeof(uint32_t);
    if (cudaMalloc(&b->d_arena, need) != cudaSuccess) {
        cudaGetLastError();
        pfb::set_error("pfb_mr: cannot allocate %zu bytes of device memory", need);
        delete b;
        return PFB_E_NOMEM;
    }
    b->d_jobs = (JobDev *)b->d_arena;
    b->d_locks = (int *)(b->d_arena + job_bytes);
    b->d_counter = (unsigned int *)(b->d_arena + job_bytes + lock_bytes - 256);
    if (mode == 2) {
        b->d_lucas = (LucasDev *)(b->d_arena + job_bytes + lock_bytes);
        b->lucas.assign(n, LucasDev{});
    }
    uint32_t *d_words = (uint32_t *)(b->d_arena + job_bytes + lock_bytes + lucas_bytes);
    if (cudaMemsetAsync(b->d_locks, 0, lock_bytes, e->stream) != cudaSuccess) {
        batch_free(b);
        return pfb::cuda_fail(cudaGetLastError(), "lock reset", __FILE__, __LINE__);
    }
    b->jobs.assign(n, JobDev{});
    size_t off = 0;
    int rc = PFB_OK;
    for (int i = 0; i < n && !rc; i++) {
        JobDev &j = b->jobs[i];
        memset(&j, 0, sizeof(j));
        const HostPrep &h = b->hp[i];
        if (!h.ok || h.decided >= 0) {
            j.phase = 3;
            j.verdict = h.ok ? h.decided : -1;
            continue;
        }
        uint32_t *w = d_words + off;
        const Layout &l = lay[i];
        j.x = w + l.x;
        j.res = w + l.res;
        j.nph = w + l.nph;
        j.nh = w + l.nh;
        j.npl = w + l.npl;
        j.nl = w + l.nl;
        j.exp = w + l.exp;
        if (h.logl > LOG_LCTA) {
            j.spill_s = w + l.ss;
            j.spill_t = w + l.st;
            j.ybuf = w + l.yb;
        }
        j.logl = h.logl;
        j.cursor = h.cursor;
        j.extra = mode >= 1 ? h.s - 1 : 0;
        j.phase = 0;
        j.base = base;
        j.mode = mode;
        const size_t H = h.x0.size();
        cudaError_t ce = cudaMemcpyAsync(j.x, h.x0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
        if (mode == 2) {
            LucasDev &lc = b->lucas[i];
            lc.lv0 = w + l.lv0;
            lc.lv1 = w + l.lv1;
            lc.lqk = w + l.lqk;
            lc.lt = w + l.lt;
            lc.lone = w + l.lone;
            lc.gy = w + l.gy;
            lc.q = h.q;
            lc.lb = h.lb;
            j.lucas = b->d_lucas + i;
            // V_0 = 2, V_1 = P = 1, Q^0 = 1, and 1 itself, in Montgomery form
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(lc.lv0, h.v0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(lc.lv1, h.x0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(lc.lqk, h.x0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(lc.lone, h.x0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
        }
        if (ce == cudaSuccess) ce = cudaMemcpyAsync((void *)j.npl, h.npl.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync((void *)j.nl, h.nl.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync((void *)j.exp, h.exp.data(), h.exp.size() * 4, cudaMemcpyHostToDevice, e->stream);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "batch upload", __FILE__, __LINE__);
        off += l.total;
    }
    cudaError_t ce = cudaSuccess;
    if (!rc) ce = cudaMemcpyAsync(b->d_jobs, b->jobs.data(), n * sizeof(JobDev), cudaMemcpyHostToDevice, e->stream);
    if (!rc && ce == cudaSuccess && mode == 2)
        ce = cudaMemcpyAsync(b->d_lucas, b->lucas.data(), n * sizeof(LucasDev), cudaMemcpyHostToDevice, e->stream);
    if (!rc && ce != cudaSuccess) rc = pfb::cuda_fail(ce, "job upload", __FILE__, __LINE__);
    if (!rc && b->n_ok) {
        prep_kernel<<<n, THREADS, smem_bytes(b->maxlog), e->stream>>>(b->d_jobs, nullptr, e->tw);
        ce = cudaGetLastError();
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "prep_kernel", __FILE__, __LINE__);
    }
    // host staging must outlive the copies; later work may use other streams
    if (!rc) {
        ce = cudaStreamSynchronize(e->stream);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "batch sync", __FILE__, __LINE__);
    }
    if (rc) {
        batch_free(b);
        return rc;
    }
    *out = b;
    return PFB_OK;
}

// Enqueues about `steps` steps of every unfinished candidate: launches of the
// persistent kernel, each handing out n * ceil(chunk / quantum) quanta.
int batch_advance(pfb_mr_batch *b, long long steps, cudaStream_t st) {
    if (!b->n_ok || steps <= 0) return PFB_OK;
    const long long cmax = b->e->chunk[b->maxlog];
    const int q0 = b->e->quantum[b->maxlog];
    while (steps > 0) {
        const long long chunk = std::min<long long>(steps, cmax);
        const int quantum = (int)std::min<long long>(chunk, q0);
        cudaGraphExec_t g = nullptr;
        const int rc = chunk_graph(b, chunk, quantum, &g);
        if (rc) return rc;
        PFB_CUDA(cudaGraphLaunch(g, st));
        steps -= chunk;
        b->steps_done += chunk;
    }
    return PFB_OK;
}

int batch_pending(pfb_mr_batch *b, int *pending, long long *steps_total) {
    PFB_CUDA(cudaStreamSynchronize(b->e->stream));
    PFB_CUDA(cudaDeviceSynchronize());
    PFB_CUDA(cudaMemcpy(b->jobs.data(), b->d_jobs, b->n * sizeof(JobDev), cudaMemcpyDeviceToHost));
    int c = 0;
    long long st = 0;
    for (int i = 0; i < b->n; i++) {
        c += b->jobs[i].phase != 3;
        st += b->jobs[i].steps;
    }
    if (pending) *pending = c;
    if (steps_total) *steps_total = st;
    return PFB_OK;
}

int batch_results(pfb_mr_batch *b, int8_t *verdict, uint16_t *residue, int residue_stride) {
    pfb_mr *e = b->e;
    PFB_CUDA(cudaMemcpyAsync(b->jobs.data(), b->d_jobs, b->n * sizeof(JobDev), cudaMemcpyDeviceToHost, e->stream));
    PFB_CUDA(cudaStreamSynchronize(e->stream));
    std::vector<uint32_t> r22;
    int rc = PFB_OK;
    for (int i = 0; i < b->n; i++) {
        const JobDev &j = b->jobs[i];
        if (!b->hp[i].ok || b->hp[i].decided >= 0) {
            if (verdict) verdict[i] = (int8_t)(b->hp[i].ok ? b->hp[i].decided : -1);
            if (residue) memset(residue + (size_t)i * residue_stride, 0, sizeof(uint16_t) * residue_stride);
            continue;
        }
        if (j.phase != 3) {
            if (verdict) verdict[i] = -2;
            rc = PFB_E_STATE;
            continue;
        }
        if (verdict) verdict[i] = (int8_t)(b->mode >= 1 ? j.verdict : 0);
        if (residue && b->mode != 2) {
            const size_t H = b->hp[i].x0.size();
            r22.resize(H);
            PFB_CUDA(cudaMemcpy(r22.data(), j.res, H * 4, cudaMemcpyDeviceToHost));
            pfb::big::Words r = pfb::big::from_limbs(r22.data(), LIMB_BITS, H);
            pfb::big::to_u16(r, residue + (size_t)i * residue_stride, (size_t)residue_stride);
        }
    }
    if (rc) pfb::set_error("pfb_mr: some candidates have not finished");
    return rc;
}

int run_jobs(pfb_mr *e, const pfb_mr_number_t *nums, int n, uint32_t base, int mode,
             const pfb_mr_number_t *exps, int8_t *verdict, uint16_t *residue, int residue_stride) {
    if (residue && residue_stride <= 0) {
        pfb::set_error("pfb_mr: residue_stride must be > 0");
        return PFB_E_ARG;
    }
    pfb_mr_batch *b = nullptr;
    int rc = batch_build(e, nums, n, base, mode, exps, &b);
    if (rc) return rc;
    rc = batch_advance(b, b->max_steps, e->stream);
    // The round-robin hands a locked candidate's quantum to another one, so a
    // few candidates may still need steps: continue until none is pending.
    // Every round advances each unfinished candidate, so a round count of
    // max_steps / 4096 + 64 is never reached unless the device stopped
    // making progress.
    const long long max_rounds = b->max_steps / 4096 + 64;
    for (long long round = 0; !rc; round++) {
        int pending = 0;
        rc = batch_pending(b, &pending, nullptr);
        if (rc || pending == 0) break;
        if (round >= max_rounds) {
            pfb::set_error("pfb_mr: %d candidates unfinished after %lld extra rounds", pending, round);
            rc = PFB_E_STATE;
            break;
        }
        rc = batch_advance(b, 4096, e->stream);
    }
    if (!rc) rc = batch_results(b, verdict, residue, residue_stride);
    cudaStreamSynchronize(e->stream);
    batch_free(b);
    return rc;
}

}  // namespace

extern "C" int pfb_mr_test(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base, int8_t *verdict,
                           uint16_t *residue, int residue_stride) {
    return run_jobs(e, nums, n, base, 1, nullptr, verdict, residue, residue_stride);
}

extern "C" int pfb_mr_lucas(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, int8_t *verdict) {
    if (!verdict) {
        pfb::set_error("pfb_mr_lucas: verdict is required");
        return PFB_E_ARG;
    }
    return run_jobs(e, nums, n, 2u, 2, nullptr, verdict, nullptr, 0);
}

extern "C" int pfb_mr_powm(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base,
                           const pfb_mr_number_t *exps, uint16_t *residue, int residue_stride) {
    if (!exps || !residue) {
        pfb::set_error("pfb_mr_powm: exps and residue are required");
        return PFB_E_ARG;
    }
    return run_jobs(e, nums, n, base, 0, exps, nullptr, residue, residue_stride);
}

extern "C" int pfb_mr_batch_create(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base,
                                   pfb_mr_batch_t **out) {
    if (!out) {
        pfb::set_error("pfb_mr_batch_create: null out");
        return PFB_E_ARG;
    }
    return batch_build(e, nums, n, base, 1, nullptr, out);
}

extern "C" int pfb_mr_batch_advance(pfb_mr_batch_t *b, int steps, void *stream) {
    if (!b || steps < 0) {
        pfb::set_error("pfb_mr_batch_advance: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(b->e->device));
    return batch_advance(b, steps, stream ? (cudaStream_t)stream : b->e->stream);
}

extern "C" int pfb_mr_batch_pending(pfb_mr_batch_t *b, int *pending) {
    if (!b || !pending) {
        pfb::set_error("pfb_mr_batch_pending: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(b->e->device));
    return batch_pending(b, pending, nullptr);
}

extern "C" long long pfb_mr_batch_steps_done(pfb_mr_batch_t *b) {
    if (!b) return -1;
    if (cudaSetDevice(b->e->device) != cudaSuccess) return -1;
    long long st = 0;
    if (batch_pending(b, nullptr, &st)) return -1;
    return st;
}

extern "C" long long pfb_mr_batch_steps_left(pfb_mr_batch_t *b) {
    if (!b) return -1;
    return std::max(0ll, b->max_steps - b->steps_done);
}

extern "C" int pfb_mr_batch_results(pfb_mr_batch_t *b, int8_t *verdict, uint16_t *residue, int residue_stride) {
    if (!b || (residue && residue_stride <= 0)) {
        pfb::set_error("pfb_mr_batch_results: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(b->e->device));
    PFB_CUDA(cudaDeviceSynchronize());
    return batch_results(b, verdict, residue, residue_stride);
}

extern "C" void pfb_mr_batch_destroy(pfb_mr_batch_t *b) {
    if (!b) return;
    cudaSetDevice(b->e->device);
    cudaDeviceSynchronize();
    batch_free(b);
}

extern "C" int pfb_mr_autotune(pfb_mr_t *e, int logl_lo, int logl_hi, pfb_mr_tune_t *results, int cap,
                               int *n_results) {
    if (!e || logl_lo < LOG_LMIN || logl_hi > LOG_LSEQ || logl_lo > logl_hi || (cap > 0 && !results)) {
        pfb::set_error("pfb_mr_autotune: bad argument (transform lengths 2^%d .. 2^%d)", LOG_LMIN, LOG_LSEQ);
        return PFB_E_ARG;
    }
    if (n_results) *n_results = 0;
    PFB_CUDA(cudaSetDevice(e->device));
    // quanta above 64 steps leave SMs idle at the end of each launch once a
    // batch holds several candidates per SM, so the search stays below
    static const int kQuanta[] = {16, 32, 64};
    static const int kChunks[] = {1024, 2048};
    constexpr int NQ = 3, NC = 2, NP = NQ * NC;
    const long long kSteps = 2048;  // timed steps per tried pair and batch shape
    const int sms = std::max(1, e->num_sms);
    int rows = 0;
    uint64_t x = 0x9E3779B97F4A7C15ull;  // xorshift64: synthetic moduli
    cudaEvent_t ev[2];
    PFB_CUDA(cudaEventCreate(&ev[0]));
    PFB_CUDA(cudaEventCreate(&ev[1]));
    int rc = PFB_OK;
    for (int lg = logl_lo; lg <= logl_hi && !rc; lg++) {
        // the longest base-2 modulus of this length: R = 2^(22 L/2) >= 2^(bits + 6)
        const size_t bits = std::min<size_t>((size_t)LIMB_BITS * ((size_t)1 << (lg - 1)) - 8, PFB_MR_MAX_BITS);
        const int n16 = (int)((bits + 15) / 16);
        const int q_old = e->quantum[lg], c_old = e->chunk[lg];
        double rate[2][NP] = {};
        // two batch shapes: one and two candidates per SM (the tail of a launch
        // weighs more with one)
        for (int shape = 0; shape < 2 && !rc; shape++) {
            const int n = (shape + 1) * sms;
            std::vector<uint16_t> limbs((size_t)n * n16);
            std::vector<pfb_mr_number_t> nums(n);
            for (int i = 0; i < n; i++) {
                uint16_t *l = limbs.data() + (size_t)i * n16;
                for (int w = 0; w < n16; w++) {
                    x ^= x << 13;
                    x ^= x >> 7;
                    x ^= x << 17;
                    l[w] = (uint16_t)x;
                }
                const int top = (int)((bits - 1) % 16);
                l[n16 - 1] = (uint16_t)((l[n16 - 1] & ((1u << top) - 1u)) | (1u << top));
                l[0] |= 1u;
                nums[i] = pfb_mr_number_t{l, n16};
            }
            pfb_mr_batch *b = nullptr;
            rc = batch_build(e, nums.data(), n, 2u, 1, nullptr, &b);
            if (rc) break;
            rc = batch_advance(b, 64, e->stream);  // warm-up
            for (int k = 0; k < NP && !rc; k++) {
                e->quantum[lg] = kQuanta[k / NC];
                e->chunk[lg] = kChunks[k % NC];
                long long before = 0, after = 0;
                rc = batch_pending(b, nullptr, &before);
                if (!rc && cudaEventRecord(ev[0], e->stream) != cudaSuccess) rc = PFB_E_CUDA;
                if (!rc) rc = batch_advance(b, kSteps, e->stream);
                if (!rc && cudaEventRecord(ev[1], e->stream) != cudaSuccess) rc = PFB_E_CUDA;
                if (!rc) rc = batch_pending(b, nullptr, &after);
                float ms = 0.f;
                if (!rc && cudaEventElapsedTime(&ms, ev[0], ev[1]) != cudaSuccess) rc = PFB_E_CUDA;
                if (!rc) rate[shape][k] = ms > 0.f ? (double)(after - before) / (1e-3 * (double)ms) : 0.0;
            }
            batch_free(b);
        }
        e->quantum[lg] = q_old;
        e->chunk[lg] = c_old;
        if (rc) break;
        // score: the sum over shapes of the rate relative to the shape's best
        double best_rate[2] = {0.0, 0.0}, best = -1.0;
        for (int shape = 0; shape < 2; shape++)
            for (int k = 0; k < NP; k++) best_rate[shape] = std::max(best_rate[shape], rate[shape][k]);
        for (int k = 0; k < NP; k++) {
            double score = 0.0;
            for (int shape = 0; shape < 2; shape++)
                score += best_rate[shape] > 0.0 ? rate[shape][k] / best_rate[shape] : 0.0;
            if (results && rows < cap)
                results[rows] = pfb_mr_tune_t{lg, kQuanta[k / NC], kChunks[k % NC], rate[0][k], rate[1][k]};
            rows++;
            if (score > best) {
                best = score;
                e->quantum[lg] = kQuanta[k / NC];
                e->chunk[lg] = kChunks[k % NC];
            }
        }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (n_results) *n_results = std::min(rows, cap);
    return rc;
}

extern "C" int pfb_mr_get_tuning(pfb_mr_t *e, int logl, int *quantum, int *chunk) {
    if (!e || logl < 0 || logl > LOG_LMAX) {
        pfb::set_error("pfb_mr_get_tuning: bad argument");
        return PFB_E_ARG;
    }
    if (quantum) *quantum = e->quantum[logl];
    if (chunk) *chunk = e->chunk[logl];
    return PFB_OK;
}

extern "C" long long pfb_mr_test_cost(const uint16_t *limbs, int n_limbs) {
    if (!limbs || n_limbs <= 0) return -1;
    pfb::big::Words N = pfb::big::from_u16(limbs, (size_t)n_limbs);
    const size_t nb = pfb::big::bit_length(N);
    if (nb < 2) return -1;
    return (long long)nb;  // ~ bits(d) squarings + one conversion
}

// ===========================================================================
// Serving: continuous batching on one GPU.
//
// Requests (candidates of any length) are prepared on host worker threads
// (N', R mod N, exponent) and admitted into free slots of a device-resident
// job table between launches of the persistent kernel, as slots and the HBM
// budget allow; every launch advances all resident candidates, whatever
// their lengths, round-robin by quanta; finished candidates are retired with
// their timestamps and their slot memory returns to a size-class pool.  All
// host waits are bounded (condition variables with timeouts); nothing on the
// device waits.

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>

namespace {

using Clock = std::chrono::steady_clock;

struct SrvRequest {
    uint64_t tag = 0;
    std::vector<uint16_t> limbs;
    uint16_t *residue_out = nullptr;
    int residue_cap = 0;
    double t_submit = 0.0, t_admit = 0.0;
    HostPrep hp;
};

struct SrvSlot {
    bool busy = false;
    int logl = 0;
    uint8_t *mem = nullptr;
    SrvRequest req;
};

}  // namespace

struct pfb_mr_server {
    pfb_mr *e = nullptr;
    pfb_mr_server_config_t cfg{};
    Clock::time_point t0;
    // device job table
    JobDev *d_jobs = nullptr;
    int *d_locks = nullptr;
    unsigned int *d_counter = nullptr;
    int *d_list = nullptr;
    uint8_t *d_table_mem = nullptr;
    std::vector<JobDev> jobs;
    std::vector<SrvSlot> slots;
    std::map<int, std::vector<uint8_t *>> pool;  // free slot memory by transform length
    size_t bytes_in_use = 0, bytes_owned = 0;
    cudaStream_t stream = nullptr;
    // queues
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<SrvRequest> submitted, prepared;
    std::deque<pfb_mr_result_t> done;
    bool stop = false;
    int preparing = 0;
    // statistics
    long long n_submitted = 0, n_admitted = 0, n_completed = 0, launches = 0;
    long long steps_total = 0;
    int resident = 0;
    std::vector<std::thread> workers;
    std::thread driver;
    int error = PFB_OK;
};

namespace {

double now_s(const pfb_mr_server *s) {
    return std::chrono::duration<double>(Clock::now() - s->t0).count();
}

size_t slot_bytes(int logl) { return slot_layout(logl).total * sizeof(uint32_t); }

void srv_prep_worker(pfb_mr_server *s) {
    for (;;) {
        SrvRequest r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            while (!s->stop && s->submitted.empty()) s->cv_work.wait_for(lk, std::chrono::milliseconds(100));
            if (s->stop) return;
            r = std::move(s->submitted.front());
            s->submitted.pop_front();
            s->preparing++;
        }
        pfb_mr_number_t num{r.limbs.data(), (int)r.limbs.size()};
        host_prep(num, s->cfg.base, 1, nullptr, r.hp);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->preparing--;
            if (!r.hp.ok) {
                pfb_mr_result_t res{};
                res.tag = r.tag;
                res.verdict = -1;
                res.submit_s = r.t_submit;
                res.admit_s = res.done_s = now_s(s);
                s->done.push_back(res);
                s->n_completed++;
                s->cv_done.notify_all();
            } else {
                s->prepared.push_back(std::move(r));
            }
        }
        s->cv_work.notify_all();
    }
}

// Admits prepared requests into free slots; returns the slots admitted.
int srv_admit(pfb_mr_server *s, std::vector<int> &admitted) {
    admitted.clear();
    for (;;) {
        SrvRequest r;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->prepared.empty()) break;
            int free_slot = -1;
            for (int i = 0; i < (int)s->slots.size(); i++)
                if (!s->slots[i].busy) {
                    free_slot = i;
                    break;
                }
            if (free_slot < 0) break;
            const int lg = s->prepared.front().hp.logl;
            const size_t need = slot_bytes(lg);
            const bool pooled = !s->pool[lg].empty();
            if (s->cfg.hbm_budget_bytes && !pooled && s->bytes_owned + need > s->cfg.hbm_budget_bytes) {
                // give back pooled blocks of other lengths first
                for (auto &kv : s->pool) {
                    while (!kv.second.empty() && s->bytes_owned + need > s->cfg.hbm_budget_bytes) {
                        const size_t blk = slot_bytes(kv.first);
                        cudaFree(kv.second.back());
                        kv.second.pop_back();
                        s->bytes_owned -= std::min(s->bytes_owned, blk);
                    }
                }
            }
            if (s->cfg.hbm_budget_bytes && !pooled && s->bytes_owned + need > s->cfg.hbm_budget_bytes) {
                if (s->resident == 0 && admitted.empty()) {
                    // a single request above the whole budget can never run
                    SrvRequest bad = std::move(s->prepared.front());
                    s->prepared.pop_front();
                    pfb_mr_result_t res{};
                    res.tag = bad.tag;
                    res.verdict = -1;
                    res.submit_s = bad.t_submit;
                    res.admit_s = res.done_s = now_s(s);
                    s->done.push_back(res);
                    s->n_completed++;
                    s->cv_done.notify_all();
                    continue;
                }
                break;  // wait for memory to come back
            }
            r = std::move(s->prepared.front());
            s->prepared.pop_front();
            SrvSlot &sl = s->slots[free_slot];
            sl.busy = true;
            sl.logl = lg;
            if (pooled) {
                sl.mem = s->pool[lg].back();
                s->pool[lg].pop_back();
            } else {
                sl.mem = nullptr;
            }
            s->bytes_in_use += need;
            admitted.push_back(free_slot);
            r.t_admit = now_s(s);
            sl.req = std::move(r);
        }
        SrvSlot &sl = s->slots[admitted.back()];
        if (!sl.mem) {
            const size_t need = slot_bytes(sl.logl);
            cudaError_t ce = cudaMalloc(&sl.mem, need);
            if (ce != cudaSuccess) {
                // the device ran out below the budget (memory held elsewhere):
                // give back the pooled blocks and try once more
                cudaGetLastError();
                std::lock_guard<std::mutex> lk(s->mu);
                for (auto &kv : s->pool) {
                    const size_t blk = slot_bytes(kv.first);
                    for (uint8_t *m : kv.second) {
                        cudaFree(m);
                        s->bytes_owned -= std::min(s->bytes_owned, blk);
                    }
                    kv.second.clear();
                }
                sl.mem = nullptr;
                ce = cudaMalloc(&sl.mem, need);
            }
            if (ce != cudaSuccess) {
                // undo the admission: the request waits for resident candidates
                // to retire, or fails if none is resident
                cudaGetLastError();
                sl.mem = nullptr;
                admitted.pop_back();
                std::lock_guard<std::mutex> lk(s->mu);
                sl.busy = false;
                s->bytes_in_use -= need;
                if (s->resident == 0 && admitted.empty()) {
                    pfb_mr_result_t res{};
                    res.tag = sl.req.tag;
                    res.verdict = -1;
                    res.submit_s = sl.req.t_submit;
                    res.admit_s = res.done_s = now_s(s);
                    s->done.push_back(res);
                    s->n_completed++;
                    s->cv_done.notify_all();
                } else {
                    s->prepared.push_front(std::move(sl.req));
                }
                sl.req = SrvRequest();
                break;
            }
            std::lock_guard<std::mutex> lk(s->mu);
            s->bytes_owned += need;
        }
        // fill the job and upload its inputs
        const HostPrep &h = sl.req.hp;
        const Layout l = slot_layout(h.logl);
        uint32_t *w = (uint32_t *)sl.mem;
        JobDev &j = s->jobs[admitted.back()];
        memset(&j, 0, sizeof(j));
        j.x = w + l.x;
        j.res = w + l.res;
        j.nph = w + l.nph;
        j.nh = w + l.nh;
        j.npl = w + l.npl;
        j.nl = w + l.nl;
        j.exp = w + l.exp;
        if (h.logl > LOG_LCTA) {
            j.spill_s = w + l.ss;
            j.spill_t = w + l.st;
            j.ybuf = w + l.yb;
        }
        j.logl = h.logl;
        j.cursor = h.cursor;
        j.extra = h.s - 1;
        j.phase = 0;
        j.base = s->cfg.base;
        j.mode = 1;
        const size_t H = h.x0.size();
        PFB_CUDA(cudaMemcpyAsync(j.x, h.x0.data(), H * 4, cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaMemcpyAsync((void *)j.npl, h.npl.data(), H * 4, cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaMemcpyAsync((void *)j.nl, h.nl.data(), H * 4, cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaMemcpyAsync((void *)j.exp, h.exp.data(), h.exp.size() * 4, cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaMemcpyAsync(s->d_jobs + admitted.back(), &j, sizeof(JobDev), cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaStreamSynchronize(s->stream));  // host staging is freed below / reused
    }
    if (!admitted.empty()) {
        PFB_CUDA(cudaMemcpyAsync(s->d_list, admitted.data(), admitted.size() * sizeof(int), cudaMemcpyHostToDevice,
                                 s->stream));
        int maxlog = LOG_LMIN;
        for (int i : admitted) maxlog = std::max(maxlog, s->slots[i].logl);
        prep_kernel<<<(int)admitted.size(), THREADS, smem_bytes(maxlog), s->stream>>>(s->d_jobs, s->d_list, s->e->tw);
        PFB_CUDA(cudaGetLastError());
        PFB_CUDA(cudaStreamSynchronize(s->stream));
        for (int i : admitted) {  // the set-up inputs are on the device now
            HostPrep &h = s->slots[i].req.hp;
            std::vector<uint32_t>().swap(h.npl);
            std::vector<uint32_t>().swap(h.exp);
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->resident += (int)admitted.size();
        s->n_admitted += (long long)admitted.size();
    }
    return PFB_OK;
}

// Retires finished candidates (host mirror of the job table already read).
void srv_retire(pfb_mr_server *s) {
    std::vector<uint32_t> r22;
    for (int i = 0; i < (int)s->slots.size(); i++) {
        SrvSlot &sl = s->slots[i];
        if (!sl.busy || s->jobs[i].phase != 3) continue;
        pfb_mr_result_t res{};
        res.tag = sl.req.tag;
        res.verdict = (int8_t)s->jobs[i].verdict;
        res.submit_s = sl.req.t_submit;
        res.admit_s = sl.req.t_admit;
        if (sl.req.residue_out && sl.req.residue_cap > 0) {
            const size_t H = sl.req.hp.x0.size();
            r22.resize(H);
            if (cudaMemcpy(r22.data(), s->jobs[i].res, H * 4, cudaMemcpyDeviceToHost) == cudaSuccess) {
                pfb::big::Words r = pfb::big::from_limbs(r22.data(), LIMB_BITS, H);
                pfb::big::to_u16(r, sl.req.residue_out, (size_t)sl.req.residue_cap);
            }
        }
        res.done_s = now_s(s);
        const size_t bytes = slot_bytes(sl.logl);
        std::lock_guard<std::mutex> lk(s->mu);
        s->pool[sl.logl].push_back(sl.mem);
        sl.mem = nullptr;
        sl.busy = false;
        s->bytes_in_use -= bytes;
        s->resident--;
        s->n_completed++;
        s->steps_total += s->jobs[i].steps;
        s->done.push_back(res);
        s->cv_done.notify_all();
    }
}

void srv_driver(pfb_mr_server *s) {
    if (cudaSetDevice(s->e->device) != cudaSuccess) {
        s->error = PFB_E_CUDA;
        return;
    }
    std::vector<int> admitted;
    const int cap = (int)s->slots.size();
    const int grid_max = std::max(1, s->e->num_sms);
    while (true) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            while (!s->stop && s->resident == 0 && s->prepared.empty())
                s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
            if (s->stop) break;
        }
        int rc = srv_admit(s, admitted);
        if (rc) {
            s->error = rc;
            break;
        }
        int res_now;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            res_now = s->resident;
        }
        if (res_now == 0) continue;
        // one launch: every resident candidate advances about chunk_steps steps
        const int quantum = std::min(64, s->cfg.chunk_steps);
        const long long qpj = (s->cfg.chunk_steps + quantum - 1) / quantum;
        int maxlog = LOG_LMIN;
        for (auto &sl : s->slots)
            if (sl.busy) maxlog = std::max(maxlog, sl.logl);
        cudaMemsetAsync(s->d_counter, 0, sizeof(unsigned int), s->stream);
        persist_kernel<<<std::min(res_now, grid_max), THREADS, smem_bytes(maxlog), s->stream>>>(
            s->d_jobs, cap, s->d_locks, s->d_counter, (unsigned int)(res_now * qpj), quantum, s->e->tw);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(s->jobs.data(), s->d_jobs, cap * sizeof(JobDev), cudaMemcpyDeviceToHost, s->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess) {
            pfb::set_error("pfb_mr_server: CUDA failure in the step loop");
            s->error = PFB_E_CUDA;
            break;
        }
        s->launches++;
        srv_retire(s);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_done.notify_all();
    s->cv_work.notify_all();
}

}  // namespace

extern "C" int pfb_mr_server_create(pfb_mr_t *e, const pfb_mr_server_config_t *cfg, pfb_mr_server_t **out) {
    if (!e || !out) {
        pfb::set_error("pfb_mr_server_create: null argument");
        return PFB_E_ARG;
    }
    *out = nullptr;
    pfb_mr_server *s = new pfb_mr_server();
    s->e = e;
    if (cfg) s->cfg = *cfg;
    if (s->cfg.max_resident <= 0) s->cfg.max_resident = 2 * std::max(1, e->num_sms);
    if (s->cfg.chunk_steps <= 0) s->cfg.chunk_steps = 512;
    if (s->cfg.base < 2 || s->cfg.base > 0xFFFFu) s->cfg.base = 2;
    if (s->cfg.prep_threads <= 0) s->cfg.prep_threads = 4;
    s->t0 = Clock::now();
    const int cap = s->cfg.max_resident;
    PFB_CUDA(cudaSetDevice(e->device));
    const size_t job_bytes = ((size_t)cap * sizeof(JobDev) + 255) & ~(size_t)255;
    const size_t int_bytes = ((size_t)cap * sizeof(int) + 255) & ~(size_t)255;
    if (cudaMalloc(&s->d_table_mem, job_bytes + 2 * int_bytes + 256) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        pfb::set_error("pfb_mr_server_create: cannot allocate the job table");
        return PFB_E_NOMEM;
    }
    s->d_jobs = (JobDev *)s->d_table_mem;
    s->d_locks = (int *)(s->d_table_mem + job_bytes);
    s->d_list = (int *)(s->d_table_mem + job_bytes + int_bytes);
    s->d_counter = (unsigned int *)(s->d_table_mem + job_bytes + 2 * int_bytes);
    s->jobs.assign(cap, JobDev{});
    for (auto &j : s->jobs) j.phase = 3;
    s->slots.resize(cap);
    int rc = PFB_OK;
    cudaError_t ce = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaMemcpy(s->d_jobs, s->jobs.data(), cap * sizeof(JobDev), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemset(s->d_locks, 0, int_bytes);
    if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "server set-up", __FILE__, __LINE__);
    if (rc) {
        cudaFree(s->d_table_mem);
        if (s->stream) cudaStreamDestroy(s->stream);
        delete s;
        return rc;
    }
    for (int t = 0; t < s->cfg.prep_threads; t++) s->workers.emplace_back(srv_prep_worker, s);
    s->driver = std::thread(srv_driver, s);
    *out = s;
    return PFB_OK;
}

extern "C" int pfb_mr_server_submit(pfb_mr_server_t *s, const uint16_t *limbs, int n_limbs, uint64_t tag,
                                    uint16_t *residue_out, int residue_cap) {
    if (!s || !limbs || n_limbs <= 0 || (residue_out && residue_cap <= 0)) {
        pfb::set_error("pfb_mr_server_submit: bad argument");
        return PFB_E_ARG;
    }
    SrvRequest r;
    r.tag = tag;
    r.limbs.assign(limbs, limbs + n_limbs);
    r.residue_out = residue_out;
    r.residue_cap = residue_cap;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            pfb::set_error("pfb_mr_server_submit: server stopped (%d)", s->error);
            return PFB_E_STATE;
        }
        r.t_submit = now_s(s);
        s->submitted.push_back(std::move(r));
        s->n_submitted++;
    }
    s->cv_work.notify_all();
    return PFB_OK;
}

extern "C" int pfb_mr_server_poll(pfb_mr_server_t *s, pfb_mr_result_t *out, int cap, int timeout_ms) {
    if (!s || !out || cap <= 0) {
        pfb::set_error("pfb_mr_server_poll: bad argument");
        return PFB_E_ARG;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && timeout_ms > 0 && !s->stop)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !s->done.empty() || s->stop; });
    int n = 0;
    while (n < cap && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    if (n == 0 && s->stop && s->error) return s->error;
    return n;
}

extern "C" int pfb_mr_server_stats(pfb_mr_server_t *s, pfb_mr_server_stats_t *st) {
    if (!s || !st) {
        pfb::set_error("pfb_mr_server_stats: bad argument");
        return PFB_E_ARG;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    st->submitted = s->n_submitted;
    st->admitted = s->n_admitted;
    st->completed = s->n_completed;
    st->resident = s->resident;
    st->queued = (int)(s->submitted.size() + s->prepared.size()) + s->preparing;
    st->launches = s->launches;
    st->steps_retired = s->steps_total;
    st->bytes_in_use = s->bytes_in_use;
    st->bytes_owned = s->bytes_owned;
    st->error = s->error;
    return PFB_OK;
}

extern "C" void pfb_mr_server_destroy(pfb_mr_server_t *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    if (s->driver.joinable()) s->driver.join();
    for (auto &t : s->workers)
        if (t.joinable()) t.join();
    cudaSetDevice(s->e->device);
    cudaStreamSynchronize(s->stream);
    for (auto &sl : s->slots)
        if (sl.mem) cudaFree(sl.mem);
    for (auto &kv : s->pool)
        for (uint8_t *m : kv.second) cudaFree(m);
    cudaFree(s->d_table_mem);
    cudaStreamDestroy(s->stream);
    delete s;
}
