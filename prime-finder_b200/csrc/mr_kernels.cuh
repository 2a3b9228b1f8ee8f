// Device side of the Miller-Rabin engine beyond the Montgomery step
// (mr_device.cuh): the per-candidate state, the set-up kernel, the exponent
// and Lucas ladders and the persistent scheduler.  Included by mr.cu; kept
// apart from the host code so that the kernels can also be compiled for the
// host and run on CPU threads in the tests.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "mr_device.cuh"

namespace pfb {
namespace mr {

__constant__ CrtConsts c_crt;

// State of one candidate in device memory.
struct JobDev {
    uint32_t *x;          // H limbs: Montgomery residue (working value)
    uint32_t *res;        // H limbs: canonical residue a^E mod N (output)
    uint32_t *nn;         // [2][H] negacyclic NTT_H(N''), N'' = -N^-1 mod (B^H + 1)
    uint32_t *nh;         // [2][H] NTT_H(N)
    const uint32_t *npl;  // H limbs of N'' (set-up input)
    const uint32_t *nl;   // H limbs of N
    const uint32_t *exp;  // exponent, 32-bit words, little-endian
    uint32_t *ybuf;       // H + H/32 words (L = 2^15 only: the residue Y, padded)
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

// Shared memory: up to L = 2^LOG_LCTA both primes' length-L transforms (A0,
// A1), the residue X and a second residue Y; at L = 2^15 three buffers of H
// padded words (A0, A1, X; every product there is of length H) and Y in the
// candidate's global ybuf.
__host__ __device__ inline size_t smem_words(int logl) {
    const size_t L = (size_t)1 << logl, H = L / 2;
    return logl <= LOG_LCTA ? 2 * (L + L / 32) + 2 * (H + H / 32) : 3 * (H + H / 32);
}
inline size_t smem_bytes(int logl) {
    return smem_words(logl) * sizeof(uint32_t) + sizeof(CarrySmem) + 16;
}

__device__ __forceinline__ void carve(uint32_t *raw, int logl, Smem &sm, uint32_t *&Y, uint32_t *ybuf) {
    const int L = 1 << logl, H = L >> 1;
    const int BA = logl <= LOG_LCTA ? L + L / 32 : H + H / 32, BX = H + H / 32;
    sm.A0 = raw;
    sm.A1 = raw + BA;
    sm.X = raw + 2 * BA;
    Y = logl <= LOG_LCTA ? sm.X + BX : ybuf;
    uintptr_t c = (uintptr_t)(raw + smem_words(logl));
    c = (c + 15) & ~(uintptr_t)15;
    sm.cs = (CarrySmem *)c;
}

// Cyclic (gc1, gc2: primes 1, 2) and negacyclic (gn1, gn2) NTT_H of the H
// limbs at src, reduced (either pair may be null); uses A0 and A1.  Together
// they are the two halves of the length-L transform of the zero-padded limbs.
template <int LOGL>
__device__ void spectra_t(const Smem &sm, const uint32_t *src, uint32_t *gc1, uint32_t *gc2, uint32_t *gn1,
                          uint32_t *gn2, const Twiddles &tw, bool cg) {
    constexpr int H = 1 << (LOGL - 1), LOGH = LOGL - 1;
    const int tid = threadIdx.x;
    for (int neg = 0; neg < 2; neg++) {
        uint32_t *g1 = neg ? gn1 : gc1, *g2 = neg ? gn2 : gc2;
        if (!g1) continue;
        for (int i = tid; i < H; i += THREADS) {
            const uint32_t v = cg ? __ldcg(src + i) : src[i];
            sm.A0[pad(i)] = v;
            sm.A1[pad(i)] = v;
        }
        __syncthreads();
        if (neg) dif_from<true, 0, LOGH, LOGH, 0, false, true>(sm.A0, sm.A1, tw);
        else dif_from<true, 0, LOGH, LOGH>(sm.A0, sm.A1, tw);
        for (int i = tid; i < H; i += THREADS) {
            g1[i] = red2(sm.A0[pad(i)], P1);
            g2[i] = red2(sm.A1[pad(i)], P2);
        }
        __syncthreads();
    }
}

#define PFB_LOGL_SWITCH(logl, CALL)                                   \
    switch (logl) {                                                   \
    case 8: { constexpr int LG = 8; CALL; } break;                    \
    case 9: { constexpr int LG = 9; CALL; } break;                    \
    case 10: { constexpr int LG = 10; CALL; } break;                  \
    case 11: { constexpr int LG = 11; CALL; } break;                  \
    case 12: { constexpr int LG = 12; CALL; } break;                  \
    case 13: { constexpr int LG = 13; CALL; } break;                  \
    case 14: { constexpr int LG = 14; CALL; } break;                  \
    case 15: { constexpr int LG = 15; CALL; } break;                  \
    }

// g[2][L] <- the spectrum of a second factor for mont_step: per prime, the
// cyclic half then the negacyclic half, of the H limbs at src, which may have
// been written earlier in the same launch (L2-coherent loads).
__device__ void spectrum(const Smem &sm, int logl, const uint32_t *src, uint32_t *g, const Twiddles &tw) {
    const int L = 1 << logl, H = L >> 1;
    PFB_LOGL_SWITCH(logl, (spectra_t<LG>(sm, src, g, g + L, g + H, g + L + H, tw, true)))
}

// Set-up of one candidate: the negacyclic spectrum of N'' (cd.nn) and the
// cyclic spectrum of N (cd.nh), each [2][H].
template <int LOGL>
__device__ void prep_t(const Smem &sm, const JobDev &jb, const Twiddles &tw) {
    constexpr int H = 1 << (LOGL - 1);
    spectra_t<LOGL>(sm, jb.npl, nullptr, nullptr, jb.nn, jb.nn + H, tw, false);
    spectra_t<LOGL>(sm, jb.nl, jb.nh, jb.nh + H, nullptr, nullptr, tw, false);
}

__global__ void __launch_bounds__(THREADS, 1) prep_kernel(JobDev *jobs, const int *list, Twiddles tw) {
    PFB_DYNAMIC_SMEM(uint32_t, raw);
    const JobDev jb = jobs[list ? list[blockIdx.x] : (int)blockIdx.x];
    if (jb.phase == 3) return;
    Smem sm;
    uint32_t *Y;
    carve(raw, jb.logl, sm, Y, jb.ybuf);
    PFB_LOGL_SWITCH(jb.logl, (prep_t<LG>(sm, jb, tw)))
}

// One Montgomery step at the candidate's transform length (gy: the spectrum
// of a second factor, see mont_step).
template <bool MUL>
__device__ __forceinline__ void mstep_t(const Smem &sm, const Cand &cd, bool square, uint32_t a, const Twiddles &tw,
                                        const uint32_t *gy) {
    PFB_LOGL_SWITCH(cd.logl, (mont_step<MUL, LG>(sm, cd, square, a, tw, c_crt, gy)))
}

// The strong test's squarings (inlined into its loop).
__device__ __forceinline__ void mstep(const Smem &sm, const Cand &cd, bool square, uint32_t a, const Twiddles &tw,
                                      const JobDev &) {
    mstep_t<false>(sm, cd, square, a, tw, nullptr);
}

// The Lucas ladder's steps: one out-of-line copy with the general product, so
// the strong test's loop keeps its own register allocation.
__device__ __noinline__ void mstep_l(const Smem &sm, const Cand &cd, bool square, uint32_t a, const Twiddles &tw,
                                     const JobDev &, const uint32_t *gy) {
    mstep_t<true>(sm, cd, square, a, tw, gy);
}

// Canonical residue of X (Montgomery form) into Y: Y = X R'^-1 mod N, X kept.
template <bool LUCAS = false>
__device__ void canonical(const Smem &sm, uint32_t *Y, const Cand &cd, const uint32_t *nl, const Twiddles &tw,
                          const JobDev &jb) {
    const int H = 1 << (cd.logl - 1);
    for (int i = threadIdx.x; i < H; i += blockDim.x) Y[pad(i)] = sm.X[pad(i)];
    __syncthreads();
    if (cd.logl <= LOG_LCTA) {  // the step runs on Y in shared memory
        Smem s2 = sm;
        s2.X = Y;
        if (LUCAS) mstep_l(s2, cd, false, 1u, tw, jb, nullptr);
        else mstep(s2, cd, false, 1u, tw, jb);
    } else {  // Y is in global memory: step on X, then exchange X and Y
        if (LUCAS) mstep_l(sm, cd, false, 1u, tw, jb, nullptr);
        else mstep(sm, cd, false, 1u, tw, jb);
        for (int i = threadIdx.x; i < H; i += blockDim.x) {
            const uint32_t t = sm.X[pad(i)];
            sm.X[pad(i)] = Y[pad(i)];
            Y[pad(i)] = t;
        }
        __syncthreads();
    }
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
    const Cand cd{jb.nn, jb.nh, jb.logl};
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
    const Cand cd{jb.nn, jb.nh, jb.logl};
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
    PFB_DYNAMIC_SMEM(uint32_t, raw);
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

}  // namespace mr
}  // namespace pfb
