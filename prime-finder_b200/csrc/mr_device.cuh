// Device arithmetic of the Miller-Rabin engine: one CTA owns one candidate and
// runs whole Montgomery squarings on chip.
//
// Replaces the reference's per-squaring chain of ~39 launches
// (batch_mod_ctx.cu:288-316 -> ntt_4step.cu:202-295 -> carry_norm.cu:63-122
// -> barrett.cu:128-199 / sub.cu:18-155) with one CTA-resident sequence of
// four length-H products (x of H limbs of 22 bits, B = 2^22, Montgomery radix
// R' = B^H + 1; see mont_step):
//
//   S = x^2 mod (B^H - 1)     cyclic NTT of length H over p1 and p2, CRT
//   D = x^2 mod (B^H + 1)     negacyclic NTT of length H
//   m = D N'' mod (B^H + 1)   negacyclic product with the stored NTT of N''
//   W = m N mod (B^H - 1)     cyclic product with the stored NTT of N
//   2 REDC(x^2) = S + W mod (B^H - 1)
//
// Exact 30-bit modular butterflies (Shoup's multiplication, Harvey's lazy
// [0, 2p) ranges) run on the integer pipe.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pfb {
namespace mr {

constexpr uint32_t P1 = 998244353u;   // 119 * 2^23 + 1, primitive root 3
constexpr uint32_t P2 = 1004535809u;  // 479 * 2^21 + 1, primitive root 3
constexpr int LIMB_BITS = 22;
constexpr uint32_t LIMB_MASK = (1u << LIMB_BITS) - 1u;
constexpr int LOG_LMAX = 15;          // twiddle tables cover L <= 2^15
constexpr int LOG_LMIN = 8;
constexpr int LOG_LCTA = 14;          // largest L whose two transforms fit one CTA
constexpr int LOG_LSEQ = 15;          // largest L of the sequential-prime step
constexpr int THREADS = 512;

// Twiddles: w[p][k] = omega^k, omega of order 2^LOG_LMAX, k < 2^(LOG_LMAX-1);
// wi = omega^-k.  *_sh are Shoup companions floor(w * 2^32 / p).
struct Twiddles {
    const uint32_t *w[2], *wsh[2], *wi[2], *wish[2];
};

// Twiddles of every radix-16 pass, regrouped per group: a pass's twiddles
// depend only on its first stage's half size h0 and the group's j0, so per
// (direction, prime, log2 h0) there are eight planes of G uint4 (G = h0/8
// groups for a forward pass, h0 for an inverse one); plane q holds twiddles
// 4q..4q+3 of group j0 at index j0 (planes 0-3 values, 4-7 Shoup
// companions).  A group reads its 15 + 15 words with 8 coalesced loads.
struct WideTabs {
    const uint4 *base;
    uint32_t off[2][2][LOG_LMAX];  // [forward/inverse][prime][log2 h0], in uint4
};
__constant__ WideTabs c_wide;

template <int DIR, int PR>
__device__ __forceinline__ void load_wide(int lh0, int j0, uint32_t *tw, uint32_t *tws) {
    const uint4 *T = c_wide.base + c_wide.off[DIR][PR][lh0];
    const int ng = DIR ? (1 << lh0) : (1 << (lh0 - 3));
    uint4 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = __ldg(T + q * ng + j0);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint32_t a[4] = {v[q].x, v[q].y, v[q].z, v[q].w};
        const uint32_t b[4] = {v[4 + q].x, v[4 + q].y, v[4 + q].z, v[4 + q].w};
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (4 * q + u < 15) {
                tw[4 * q + u] = a[u];
                tws[4 * q + u] = b[u];
            }
    }
}

// Per transform length (index logn): sigma = 2^32 / n mod p (undoes the
// Montgomery factor of the pointwise product and the 1/n of the inverse).
struct CrtConsts {
    uint32_t s1[LOG_LMAX + 1], s1sh[LOG_LMAX + 1];   // sigma mod p1
    uint32_t k2[LOG_LMAX + 1], k2sh[LOG_LMAX + 1];   // sigma * p1^-1 mod p2
    uint32_t k1, k1sh;                               // p1^-1 mod p2
    uint32_t pinv[2];                                // -p^-1 mod 2^32
};

__device__ __forceinline__ int pad(int i) { return i + (i >> 5); }

__device__ __forceinline__ uint32_t shoup(uint32_t a, uint32_t w, uint32_t wsh, uint32_t p) {
    const uint32_t q = __umulhi(a, wsh);
    return a * w - q * p;  // in [0, 2p) for a < 2^32
}

__device__ __forceinline__ uint32_t mont(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    const uint32_t lo = a * b, hi = __umulhi(a, b);
    const uint32_t m = lo * pinv;
    return hi + __umulhi(m, p) + (lo != 0u);  // in [0, 2p) for a, b < 2p
}

__device__ __forceinline__ uint32_t red2(uint32_t x, uint32_t p2) { return x >= p2 ? x - p2 : x; }

// Twiddles of one radix-2^RLOG group: stage s uses omega_{2 hs}^j for
// j = j0 + e * sub (DIF) or j0 + e * h0 (DIT), e < 2^s or 2^(RLOG-1-s).
template <int RLOG, bool DIT>
__device__ __forceinline__ void load_tw(const uint32_t *__restrict__ W, const uint32_t *__restrict__ Wsh, int j0,
                                        int step, int lh0, uint32_t *tw, uint32_t *tws) {
    constexpr int R = 1 << RLOG;
#pragma unroll
    for (int s = 0, t = 0; s < RLOG; s++) {
        const int cnt = DIT ? (1 << s) : (R >> (s + 1));
        const int shift = DIT ? LOG_LMAX - 1 - (lh0 + s) : LOG_LMAX - 1 - (lh0 - s);
#pragma unroll
        for (int e = 0; e < cnt; e++, t++) {
            const int k = (j0 + e * step) << shift;
            tw[t] = __ldg(W + k);
            tws[t] = __ldg(Wsh + k);
        }
    }
}

// ----- radix-2^RLOG passes --------------------------------------------------
// Decimation in frequency forward (natural order in, bit-reversed out after
// all passes), decimation in time inverse (bit-reversed in, natural out).
// log2 of the length, of the first stage's half size h0 and of the thread
// stride are template arguments, so group counts and strides are constants
// and, for element strides that are multiples of 32, so are the padded
// element offsets inside a group.  When every group of a thread has the same
// j0 (all passes but the widest) its twiddles are loaded once per pass.

// ZHI: the group's upper half (e >= R/2) is known to be zero and is not read;
// the lower half holds limbs (< 2p), so the first stage is x, x w.  The lower
// half is read from src when given (same padded layout), else from A.
// TSH > 0: the elements are first twisted for a negacyclic transform,
// element i multiplied by psi^i = ww[i << (TSH - 1)] (Shoup companion wwsh).
template <int PR, int RLOG, int SUB, bool ZHI = false, int TSH = 0>
__device__ __forceinline__ void dif_group_t(uint32_t *__restrict__ A, int base, const uint32_t *tw,
                                            const uint32_t *tws, const uint32_t *__restrict__ ww = nullptr,
                                            const uint32_t *__restrict__ wwsh = nullptr,
                                            const uint32_t *src = nullptr) {
    constexpr int R = 1 << RLOG, NL = ZHI ? R / 2 : R;
    constexpr uint32_t p = PR ? P2 : P1, p2 = 2u * p;
    const uint32_t *in = (ZHI && src) ? src : A;
    uint32_t v[R];
    if constexpr (SUB % 32 == 0) {
        constexpr int PS = SUB + SUB / 32;  // pad(base + e SUB) = pad(base) + e PS
        const int pb = pad(base);
#pragma unroll
        for (int e = 0; e < NL; e++) v[e] = in[pb + e * PS];
    } else {
#pragma unroll
        for (int e = 0; e < NL; e++) v[e] = in[pad(base + e * SUB)];
    }
    if constexpr (TSH > 0) {
#pragma unroll
        for (int e = 0; e < NL; e++) {
            const int k = (base + e * SUB) << (TSH - 1);
            v[e] = shoup(v[e], __ldg(ww + k), __ldg(wwsh + k), p);
        }
    }
#pragma unroll
    for (int s = 0, t0 = 0; s < RLOG; t0 += R >> (s + 1), s++) {
        const int half = R >> (s + 1);
#pragma unroll
        for (int e = 0; e < R; e++) {
            if (e & half) continue;
            const int t = t0 + (e & (half - 1));
            if (ZHI && s == 0) {
                v[e + half] = shoup(v[e], tw[t], tws[t], p);
                continue;
            }
            const uint32_t x = v[e], y = v[e + half];
            v[e] = red2(x + y, p2);
            v[e + half] = shoup(x - y + p2, tw[t], tws[t], p);
        }
    }
    if constexpr (SUB % 32 == 0) {
        constexpr int PS = SUB + SUB / 32;
        const int pb = pad(base);
#pragma unroll
        for (int e = 0; e < R; e++) A[pb + e * PS] = v[e];
    } else {
#pragma unroll
        for (int e = 0; e < R; e++) A[pad(base + e * SUB)] = v[e];
    }
}

// TSH > 0: the results are untwisted, element i multiplied by
// psi^-i = ww[i << (TSH - 1)] (the inverse of a negacyclic transform).
template <int PR, int RLOG, int H0, int TSH = 0>
__device__ __forceinline__ void dit_group_t(uint32_t *__restrict__ A, int base, const uint32_t *tw,
                                            const uint32_t *tws, const uint32_t *__restrict__ ww = nullptr,
                                            const uint32_t *__restrict__ wwsh = nullptr) {
    constexpr int R = 1 << RLOG;
    constexpr uint32_t p = PR ? P2 : P1, p2 = 2u * p;
    uint32_t v[R];
    if constexpr (H0 % 32 == 0) {
        constexpr int PS = H0 + H0 / 32;
        const int pb = pad(base);
#pragma unroll
        for (int e = 0; e < R; e++) v[e] = A[pb + e * PS];
    } else {
#pragma unroll
        for (int e = 0; e < R; e++) v[e] = A[pad(base + e * H0)];
    }
#pragma unroll
    for (int s = 0, t0 = 0; s < RLOG; t0 += 1 << s, s++) {
        const int half = 1 << s;
#pragma unroll
        for (int e = 0; e < R; e++) {
            if (e & half) continue;
            const int t = t0 + (e & (half - 1));
            const uint32_t x = v[e];
            const uint32_t u = shoup(v[e + half], tw[t], tws[t], p);
            v[e] = red2(x + u, p2);
            v[e + half] = red2(x - u + p2, p2);
        }
    }
    if constexpr (TSH > 0) {
#pragma unroll
        for (int e = 0; e < R; e++) {
            const int k = (base + e * H0) << (TSH - 1);
            v[e] = shoup(v[e], __ldg(ww + k), __ldg(wwsh + k), p);
        }
    }
    if constexpr (H0 % 32 == 0) {
        constexpr int PS = H0 + H0 / 32;
        const int pb = pad(base);
#pragma unroll
        for (int e = 0; e < R; e++) A[pb + e * PS] = v[e];
    } else {
#pragma unroll
        for (int e = 0; e < R; e++) A[pad(base + e * H0)] = v[e];
    }
}

template <int PR, int RLOG, int LOGN, int LH0, int STRIDE, bool ZHI = false, int TSH = 0>
__device__ __forceinline__ void dif_pass_t(uint32_t *__restrict__ A, const uint32_t *__restrict__ W,
                                           const uint32_t *__restrict__ Wsh, int g0,
                                           const uint32_t *__restrict__ ww = nullptr,
                                           const uint32_t *__restrict__ wwsh = nullptr,
                                           const uint32_t *src = nullptr) {
    constexpr int R = 1 << RLOG, H0 = 1 << LH0;
    constexpr int GROUPS = (1 << LOGN) >> RLOG;
    constexpr int SUB = (2 * H0) >> RLOG;
    uint32_t ta[R - 1], tsa[R - 1];
    if constexpr (STRIDE % SUB == 0) {  // every group of this thread has the same j0
        if constexpr (RLOG == 4) load_wide<0, PR>(LH0, g0 % SUB, ta, tsa);
        else load_tw<RLOG, false>(W, Wsh, g0 % SUB, SUB, LH0, ta, tsa);
#pragma unroll 1
        for (int gg = g0; gg < GROUPS; gg += STRIDE) {
            const int block = gg / SUB, j0 = gg % SUB;
            dif_group_t<PR, RLOG, SUB, ZHI, TSH>(A, block * 2 * H0 + j0, ta, tsa, ww, wwsh, src);
        }
    } else {
#pragma unroll 1
        for (int gg = g0; gg < GROUPS; gg += STRIDE) {
            const int block = gg / SUB, j0 = gg % SUB;
            if constexpr (RLOG == 4) load_wide<0, PR>(LH0, j0, ta, tsa);
            else load_tw<RLOG, false>(W, Wsh, j0, SUB, LH0, ta, tsa);
            dif_group_t<PR, RLOG, SUB, ZHI, TSH>(A, block * 2 * H0 + j0, ta, tsa, ww, wwsh, src);
        }
    }
}

template <int PR, int RLOG, int LOGN, int LH0, int STRIDE, int TSH = 0>
__device__ __forceinline__ void dit_pass_t(uint32_t *__restrict__ A, const uint32_t *__restrict__ W,
                                           const uint32_t *__restrict__ Wsh, int g0,
                                           const uint32_t *__restrict__ ww = nullptr,
                                           const uint32_t *__restrict__ wwsh = nullptr) {
    constexpr int R = 1 << RLOG, H0 = 1 << LH0;
    constexpr int GROUPS = (1 << LOGN) >> RLOG;
    uint32_t ta[R - 1], tsa[R - 1];
    if constexpr (STRIDE % H0 == 0) {
        if constexpr (RLOG == 4) load_wide<1, PR>(LH0, g0 & (H0 - 1), ta, tsa);
        else load_tw<RLOG, true>(W, Wsh, g0 & (H0 - 1), H0, LH0, ta, tsa);
#pragma unroll 1
        for (int gg = g0; gg < GROUPS; gg += STRIDE) {
            const int j0 = gg & (H0 - 1);
            dit_group_t<PR, RLOG, H0, TSH>(A, (gg >> LH0) * R * H0 + j0, ta, tsa, ww, wwsh);
        }
    } else {
#pragma unroll 1
        for (int gg = g0; gg < GROUPS; gg += STRIDE) {
            const int j0 = gg & (H0 - 1);
            if constexpr (RLOG == 4) load_wide<1, PR>(LH0, j0, ta, tsa);
            else load_tw<RLOG, true>(W, Wsh, j0, H0, LH0, ta, tsa);
            dit_group_t<PR, RLOG, H0, TSH>(A, (gg >> LH0) * R * H0 + j0, ta, tsa, ww, wwsh);
        }
    }
}

// Forward passes from S remaining stages down (h0 = 2^(S-1)); two primes
// split the CTA (TWO) or one prime uses all of it.  ZHI (first pass only,
// S = LOGN): the input's upper half is zero and is neither read nor stored
// beforehand (a zero-padded operand of a full-length product).  NEG: a
// negacyclic transform, the first pass twisting its inputs by psi^i (psi a
// primitive 2^(LOGN+1)-th root of unity).
template <bool TWO, int PR, int LOGN, int S, int STOP = 0, bool ZHI = false, bool NEG = false>
__device__ __forceinline__ void dif_from(uint32_t *A0, uint32_t *A1, const Twiddles &tw,
                                         const uint32_t *src = nullptr) {
    static_assert(!ZHI || (S == LOGN && S >= 4), "ZHI: first radix-16 pass of the transform");
    static_assert(!NEG || (S == LOGN && S > STOP && LOGN < LOG_LMAX), "NEG: a forward pass to twist in");
    if constexpr (S > STOP) {
        constexpr int RLOG = S >= 4 ? 4 : S;
        constexpr int TSH = NEG ? LOG_LMAX - LOGN : 0;  // shift + 1
        if constexpr (TWO) {
            constexpr int half = THREADS / 2;
            if ((int)threadIdx.x < half)
                dif_pass_t<0, RLOG, LOGN, S - 1, half, ZHI, TSH>(A0, tw.w[0], tw.wsh[0], threadIdx.x, tw.w[0],
                                                                  tw.wsh[0], src);
            else
                dif_pass_t<1, RLOG, LOGN, S - 1, half, ZHI, TSH>(A1, tw.w[1], tw.wsh[1], threadIdx.x - half, tw.w[1],
                                                                  tw.wsh[1], src);
        } else {
            dif_pass_t<PR, RLOG, LOGN, S - 1, THREADS, ZHI, TSH>(A0, tw.w[PR], tw.wsh[PR], threadIdx.x, tw.w[PR],
                                                                  tw.wsh[PR], src);
        }
        __syncthreads();
        dif_from<TWO, PR, LOGN, S - RLOG, STOP>(A0, A1, tw);
    }
}

// Inverse passes from h0 = 2^LH0 up; the remainder pass (LOGN mod 4) first.
// NEG: the last pass untwists its results by psi^-i.
template <bool TWO, int PR, int LOGN, int LH0, bool NEG = false>
__device__ __forceinline__ void dit_from(uint32_t *A0, uint32_t *A1, const Twiddles &tw) {
    if constexpr (LH0 < LOGN) {
        constexpr int RLOG = (LH0 == 0 && (LOGN & 3)) ? (LOGN & 3) : 4;
        constexpr int TSH = (NEG && LH0 + RLOG == LOGN) ? LOG_LMAX - LOGN : 0;
        if constexpr (TWO) {
            constexpr int half = THREADS / 2;
            if ((int)threadIdx.x < half)
                dit_pass_t<0, RLOG, LOGN, LH0, half, TSH>(A0, tw.wi[0], tw.wish[0], threadIdx.x, tw.wi[0], tw.wish[0]);
            else
                dit_pass_t<1, RLOG, LOGN, LH0, half, TSH>(A1, tw.wi[1], tw.wish[1], threadIdx.x - half, tw.wi[1],
                                                           tw.wish[1]);
        } else {
            dit_pass_t<PR, RLOG, LOGN, LH0, THREADS, TSH>(A0, tw.wi[PR], tw.wish[PR], threadIdx.x, tw.wi[PR],
                                                          tw.wish[PR]);
        }
        __syncthreads();
        dit_from<TWO, PR, LOGN, LH0 + RLOG, NEG>(A0, A1, tw);
    }
}

// Radix of the last forward pass, which is also the first inverse pass: both
// act on groups of R = 2^MID_RLOG consecutive elements with one twiddle set.
template <int LOGN>
constexpr int mid_rlog() {
    return (LOGN & 3) ? (LOGN & 3) : 4;
}

// The last forward pass, the pointwise product and the first inverse pass in
// one sweep over those groups (the three would otherwise each read and write
// the whole transform in shared memory).  OP 0: square; OP 1: Montgomery
// product with C (L2-coherent loads when CG: written in the same launch).
template <int PR, int LOGN, int OP, bool CG, int STRIDE>
__device__ __forceinline__ void mid_pass_t(uint32_t *__restrict__ A, const Twiddles &tw,
                                           const uint32_t *__restrict__ C, int g0, const CrtConsts &cc) {
    constexpr int RLOG = mid_rlog<LOGN>(), R = 1 << RLOG;
    constexpr int GROUPS = (1 << LOGN) >> RLOG;
    constexpr uint32_t p = PR ? P2 : P1, p2 = 2u * p;
    uint32_t ta[R - 1], tsa[R - 1], tb[R - 1], tsb[R - 1];
    if constexpr (RLOG == 4) {
        load_wide<0, PR>(RLOG - 1, 0, ta, tsa);
        load_wide<1, PR>(0, 0, tb, tsb);
    } else {
        load_tw<RLOG, false>(tw.w[PR], tw.wsh[PR], 0, 1, RLOG - 1, ta, tsa);
        load_tw<RLOG, true>(tw.wi[PR], tw.wish[PR], 0, 1, 0, tb, tsb);
    }
#pragma unroll 1
    for (int gg = g0; gg < GROUPS; gg += STRIDE) {
        const int base = gg * R, pb = pad(base);  // R | 32: the group shares one pad offset
        uint32_t v[R];
#pragma unroll
        for (int e = 0; e < R; e++) v[e] = A[pb + e];
#pragma unroll
        for (int s = 0, t0 = 0; s < RLOG; t0 += R >> (s + 1), s++) {  // forward, sub = 1
            const int half = R >> (s + 1);
#pragma unroll
            for (int e = 0; e < R; e++) {
                if (e & half) continue;
                const int t = t0 + (e & (half - 1));
                const uint32_t x = v[e], y = v[e + half];
                v[e] = red2(x + y, p2);
                v[e + half] = shoup(x - y + p2, ta[t], tsa[t], p);
            }
        }
        if constexpr (OP == 0) {
#pragma unroll
            for (int e = 0; e < R; e++) v[e] = mont(v[e], v[e], p, cc.pinv[PR]);
        } else {
#pragma unroll
            for (int e = 0; e < R; e++) v[e] = mont(v[e], CG ? __ldcg(C + base + e) : __ldg(C + base + e), p, cc.pinv[PR]);
        }
#pragma unroll
        for (int s = 0, t0 = 0; s < RLOG; t0 += 1 << s, s++) {  // inverse, h0 = 1
            const int half = 1 << s;
#pragma unroll
            for (int e = 0; e < R; e++) {
                if (e & half) continue;
                const int t = t0 + (e & (half - 1));
                const uint32_t x = v[e];
                const uint32_t u = shoup(v[e + half], tb[t], tsb[t], p);
                v[e] = red2(x + u, p2);
                v[e + half] = red2(x - u + p2, p2);
            }
        }
#pragma unroll
        for (int e = 0; e < R; e++) A[pb + e] = v[e];
    }
}

// Forward transform, pointwise product and inverse transform of length
// 2^LOGN: all forward passes but the last, the fused middle sweep, all
// inverse passes but the first.  C0/C1: the stored spectra of the two primes
// (OP 1).  ZHI: the operand's upper half is zero and was never stored.
// NEG: negacyclic (twist in the first forward pass, untwist in the last
// inverse pass; needs at least one pass on each side of the middle sweep).
template <bool TWO, int PR, int LOGN, int OP, bool CG, bool ZHI = false, bool NEG = false>
__device__ __forceinline__ void product_from(uint32_t *A0, uint32_t *A1, const Twiddles &tw, const uint32_t *C0,
                                             const uint32_t *C1, const CrtConsts &cc,
                                             const uint32_t *src = nullptr) {
    constexpr int M = mid_rlog<LOGN>();
    dif_from<TWO, PR, LOGN, LOGN, M, ZHI, NEG>(A0, A1, tw, src);
    if constexpr (TWO) {
        constexpr int half = THREADS / 2;
        if ((int)threadIdx.x < half) mid_pass_t<0, LOGN, OP, CG, half>(A0, tw, C0, threadIdx.x, cc);
        else mid_pass_t<1, LOGN, OP, CG, half>(A1, tw, C1, threadIdx.x - half, cc);
    } else {
        mid_pass_t<PR, LOGN, OP, CG, THREADS>(A0, tw, C0, threadIdx.x, cc);
    }
    __syncthreads();
    dit_from<TWO, PR, LOGN, M, NEG>(A0, A1, tw);
}

#define PFB_LOGN_CASES(F) \
    F(7) F(8) F(9) F(10) F(11) F(12) F(13) F(14) F(15)

__device__ void dif(uint32_t *A0, uint32_t *A1, int logn, const Twiddles &tw) {
    switch (logn) {
#define PFB_CASE(n)                                  \
    case n:                                          \
        dif_from<true, 0, n, n>(A0, A1, tw);         \
        return;
        PFB_LOGN_CASES(PFB_CASE)
#undef PFB_CASE
    }
}

__device__ void dit(uint32_t *A0, uint32_t *A1, int logn, const Twiddles &tw) {
    switch (logn) {
#define PFB_CASE(n)                                  \
    case n:                                          \
        dit_from<true, 0, n, 0>(A0, A1, tw);         \
        return;
        PFB_LOGN_CASES(PFB_CASE)
#undef PFB_CASE
    }
}

// Single-prime transforms: all threads of the CTA work on prime PR.
template <int PR>
__device__ void dif1(uint32_t *A, int logn, const Twiddles &tw) {
    switch (logn) {
#define PFB_CASE(n)                                  \
    case n:                                          \
        dif_from<false, PR, n, n>(A, nullptr, tw);   \
        return;
        PFB_LOGN_CASES(PFB_CASE)
#undef PFB_CASE
    }
}

template <int PR>
__device__ void dit1(uint32_t *A, int logn, const Twiddles &tw) {
    switch (logn) {
#define PFB_CASE(n)                                  \
    case n:                                          \
        dit_from<false, PR, n, 0>(A, nullptr, tw);   \
        return;
        PFB_LOGN_CASES(PFB_CASE)
#undef PFB_CASE
    }
}

// Scratch of the carry-lookahead scan.
struct CarrySmem {
    unsigned long long wc[THREADS / 32];
    uint32_t wg[THREADS / 32], wp[THREADS / 32];
    uint32_t flag;
};

// Turns n raw coefficients get(i) (each < 2^63 - 2^42) plus a carry cin0 at
// position 0 into n limbs of 22 bits written to out[] (padded index when
// PAD), and returns the carry out of position n-1 (n >= 128, a power of
// two).  Each thread propagates a segment of n/T consecutive positions; the
// carries between segments are resolved by a generate/propagate scan (warp
// ballots, then every warp over the warp aggregates): three block barriers.
template <bool PAD, class Get>
__device__ __forceinline__ unsigned long long carry_pass(const int n, const unsigned long long cin0, Get get,
                                                         uint32_t *out, CarrySmem &cs) {
    constexpr int T = THREADS;  // every kernel of the engine runs THREADS threads per CTA
    const int w = n >= 2 * T ? n / T : 2;  // >= 2 limbs: a carry-in (< 2^41) never overflows a segment twice
    const int na = n / w;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const unsigned FULL = 0xffffffffu;
    unsigned long long acc = 0, room = ~0ull;
    if (t < na) {
        const int lo = t * w;
        uint32_t l0 = 0, l1 = 0;
        bool ones = true;
        for (int q = 0; q < w; q += 2) {  // w is even
            unsigned long long vv[2];
#pragma unroll
            for (int u = 0; u < 2; u++) vv[u] = get(lo + q + u);
#pragma unroll
            for (int u = 0; u < 2; u++) {
                acc += vv[u];
                const uint32_t limb = (uint32_t)acc & LIMB_MASK;
                acc >>= LIMB_BITS;
                out[PAD ? pad(lo + q + u) : lo + q + u] = limb;
                if (q + u == 0) l0 = limb;
                else if (q + u == 1) l1 = limb;
                else ones = ones && (limb == LIMB_MASK);
            }
        }
        if (ones) room = (1ull << (2 * LIMB_BITS)) - ((unsigned long long)l1 << LIMB_BITS) - l0;
    }
    unsigned long long prev = __shfl_up_sync(FULL, acc, 1);
    if (lane == 31) cs.wc[warp] = acc;
    __syncthreads();
    if (lane == 0) prev = (warp == 0) ? cin0 : cs.wc[warp - 1];
    const bool G = (t < na) && (prev >= room);
    const bool Pr = (t < na) && !G && (prev + 1ull == room);
    const uint32_t g = __ballot_sync(FULL, G), p = __ballot_sync(FULL, Pr);
    const unsigned long long gp = (unsigned long long)(g | p);
    if (lane == 0) {
        const uint32_t o0 = (uint32_t)(((unsigned long long)g + gp) >> 32);
        const uint32_t o1 = (uint32_t)(((unsigned long long)g + gp + 1ull) >> 32);
        cs.wg[warp] = o0;
        cs.wp[warp] = o1 & (o0 ^ 1u);
    }
    __syncthreads();
    // Every warp scans the warp aggregates itself: bit v of cw is the carry
    // into warp v (v <= nw: the carry out of the last warp is bit nw).
    constexpr int nw = T / 32;
    static_assert(nw < 32, "one ballot holds the warp aggregates");
    const uint32_t G2 = __ballot_sync(FULL, lane < nw && cs.wg[lane]);
    const uint32_t P2m = __ballot_sync(FULL, lane < nw && cs.wp[lane]);
    const uint32_t cw = (uint32_t)((unsigned long long)G2 + (unsigned long long)(G2 | P2m)) ^ P2m;
    const uint32_t X = (uint32_t)((unsigned long long)g + gp + ((cw >> warp) & 1u));
    const uint32_t dprev = ((X ^ p) >> lane) & 1u;
    const unsigned long long cin = prev + dprev;
    if (t < na && cin) {
        const int lo = t * w;
        unsigned long long a2 = cin;
        for (int q = 0; q < w && a2; q++) {
            const int ix = PAD ? pad(lo + q) : lo + q;
            a2 += out[ix];
            out[ix] = (uint32_t)a2 & LIMB_MASK;
            a2 >>= LIMB_BITS;
        }
    }
    // na is a multiple of 32 (n >= 64, a power of two): the last segment is
    // lane 31 of warp na/32 - 1, its carry-out the carry into warp na/32.
    const int wl = na >> 5;
    const unsigned long long tot = cs.wc[wl - 1] + ((cw >> wl) & 1u);
    __syncthreads();
    return tot;
}

__device__ __forceinline__ unsigned long long crt(uint32_t r1, uint32_t r2, int logn, const CrtConsts &cc) {
    uint32_t c1 = shoup(r1, cc.s1[logn], cc.s1sh[logn], P1);
    c1 = red2(c1, P1);
    const uint32_t a = shoup(r2, cc.k2[logn], cc.k2sh[logn], P2);
    const uint32_t b = shoup(c1, cc.k1, cc.k1sh, P2);
    uint32_t t = a + 2u * P2 - b;  // (0, 4 p2)
    t = red2(t, 2u * P2);
    t = red2(t, P2);
    return (unsigned long long)c1 + (unsigned long long)P1 * t;
}

// Pointwise Montgomery product of a transform in shared memory with a stored
// spectrum in global memory (16-byte loads, 4 consecutive points per thread).
template <int PR, bool CG = false>
__device__ __forceinline__ void pointwise1(uint32_t *A, const uint32_t *__restrict__ C, int n, const CrtConsts &cc) {
    constexpr uint32_t p = PR ? P2 : P1;
    const uint4 *C4 = reinterpret_cast<const uint4 *>(C);
    for (int i4 = threadIdx.x; i4 < (n >> 2); i4 += blockDim.x) {
        const uint4 c = CG ? __ldcg(C4 + i4) : __ldg(C4 + i4);
        const int i = 4 * i4;
        A[pad(i)] = mont(A[pad(i)], c.x, p, cc.pinv[PR]);
        A[pad(i + 1)] = mont(A[pad(i + 1)], c.y, p, cc.pinv[PR]);
        A[pad(i + 2)] = mont(A[pad(i + 2)], c.z, p, cc.pinv[PR]);
        A[pad(i + 3)] = mont(A[pad(i + 3)], c.w, p, cc.pinv[PR]);
    }
    __syncthreads();
}

// CG: the operand was written earlier in the same launch (L2-coherent loads).
template <bool CG = false>
__device__ __forceinline__ void pointwise2(uint32_t *A0, uint32_t *A1, const uint32_t *__restrict__ C0,
                                           const uint32_t *__restrict__ C1, int n, const CrtConsts &cc) {
    const uint4 *C04 = reinterpret_cast<const uint4 *>(C0);
    const uint4 *C14 = reinterpret_cast<const uint4 *>(C1);
    for (int i4 = threadIdx.x; i4 < (n >> 2); i4 += blockDim.x) {
        const uint4 c = CG ? __ldcg(C04 + i4) : __ldg(C04 + i4);
        const uint4 d = CG ? __ldcg(C14 + i4) : __ldg(C14 + i4);
        const int i = 4 * i4;
        A0[pad(i)] = mont(A0[pad(i)], c.x, P1, cc.pinv[0]);
        A0[pad(i + 1)] = mont(A0[pad(i + 1)], c.y, P1, cc.pinv[0]);
        A0[pad(i + 2)] = mont(A0[pad(i + 2)], c.z, P1, cc.pinv[0]);
        A0[pad(i + 3)] = mont(A0[pad(i + 3)], c.w, P1, cc.pinv[0]);
        A1[pad(i)] = mont(A1[pad(i)], d.x, P2, cc.pinv[1]);
        A1[pad(i + 1)] = mont(A1[pad(i + 1)], d.y, P2, cc.pinv[1]);
        A1[pad(i + 2)] = mont(A1[pad(i + 2)], d.z, P2, cc.pinv[1]);
        A1[pad(i + 3)] = mont(A1[pad(i + 3)], d.w, P2, cc.pinv[1]);
    }
    __syncthreads();
}

// Per-CTA view of one candidate.
struct Cand {
    const uint32_t *nn;    // NTT of N'' = -N^-1 mod (B^H + 1), negacyclic, [2][H]
    const uint32_t *nh;    // NTT_H(N), cyclic, [2][H]
    int logl;
};

// Shared-memory view of one step: transform buffers A0, A1 (L padded words
// each up to L = 2^LOG_LCTA, H above), the residue X (H padded words) and
// the carry scratch.
struct Smem {
    uint32_t *A0, *A1, *X;
    CarrySmem *cs;
};

// Signed coefficients.  A product of two H-coefficient operands with limbs in
// (-2^22, 2^22 + 2) has coefficients c with |c| < H 2^44 (1 + 2^-20) < P12/2
// (H <= 2^14); the CRT gives c mod P12.  Adding OFF_i >= 2^59 - 2^37 to
// position i makes every coefficient non-negative for the carry pass, and
// the offsets sum to a multiple of the modulus the product lives in:
//   cyclic (mod B^H - 1):     OFF_i = 2^37 (B - 1)                sum 2^37 (B^H - 1)
//   negacyclic (mod B^H + 1): OFF_0 = 2^37 (B + 1), OFF_i = 2^37 (B - 1)   sum 2^37 (B^H + 1)
constexpr unsigned long long P12 = (unsigned long long)P1 * P2;
constexpr unsigned long long OFF_C = (1ull << 37) * ((1ull << LIMB_BITS) - 1ull);
constexpr unsigned long long OFF_N0 = (1ull << 37) * ((1ull << LIMB_BITS) + 1ull);

__device__ __forceinline__ unsigned long long crt_signed(uint32_t r1, uint32_t r2, int logn, const CrtConsts &cc,
                                                         unsigned long long off) {
    const unsigned long long v = crt(r1, r2, logn, cc);
    return v + off - (v > P12 / 2 ? P12 : 0ull);
}

// One Montgomery step on X (H limbs of 22 bits), with the Montgomery radix
// R' = B^H + 1 (B = 2^22):
//   X <- REDC(X^2) * a      (square = true)
//   X <- REDC(X * Y) * a    (gy = spectrum of Y, the length-L transform of its
//                            zero-padded limbs: cyclic half, negacyclic half)
//   X <- REDC(X) * a        (square = false, no gy)
// REDC(T) = (T + m N) / R' with m = -T N^-1 mod R' in [0, R'):
//   S = T mod (B^H - 1),  D = T mod (B^H + 1)
//   m = D N'' mod (B^H + 1)   negacyclic product with the stored spectrum of N''
//   W = m N mod (B^H - 1)     cyclic product with the stored spectrum of N
//   V = S + W mod (B^H - 1)
// Up to L = 2^LOG_LCTA, T comes from one zero-padded length-L product, S and
// D from its halves (S = T_lo + T_hi, D = T_lo - T_hi, no carry needed for D);
// at L = 2^15 both primes of a length-L transform do not fit one CTA, so S and
// D come from a cyclic and a negacyclic product of length H (the two halves of
// that transform, computed apart).  Since R' == 2 (mod B^H - 1), V == 2U for
// U = REDC(T); U < 2N and 4N < B^H - 1 make V = 2U exactly, so a U is (a/2) V
// for even a (the base-2 ladder's multiply by 2 costs nothing) and a (V >> 1)
// for odd a.  That is 4 length-L-equivalent transforms per step where the
// radix B^H needs 5 (its m = (T mod B^H) N' mod B^H is a zero-padded
// length-L product).
// On entry X, Y < c N with R' > 4 c^2 N (c = 4 for the strong test), or
// X < R' for a plain REDC; on exit X < 2N * a.  A0 and A1 are clobbered.
// X <- X + c mod B^H - 1 for the end-around carry c < 2^44 of a carry pass:
// warp 0 adds c to limbs 0..31 with a ballot carry-lookahead; only when the
// sum carries out of limb 31 (limbs 2..31 all B - 1) do full carry passes
// take over.
__device__ __forceinline__ void end_around(uint32_t *X, unsigned long long c, int H, CarrySmem &cs) {
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid < 32) {
        const uint32_t add = lane == 0 ? (uint32_t)c & LIMB_MASK : (lane == 1 ? (uint32_t)(c >> LIMB_BITS) : 0u);
        const uint32_t a = X[pad(lane)] + add;                  // < 2^23
        const uint32_t limb = a & LIMB_MASK;
        const uint32_t g = __ballot_sync(0xffffffffu, a > LIMB_MASK);
        const uint32_t p = __ballot_sync(0xffffffffu, a <= LIMB_MASK && limb == LIMB_MASK);
        const unsigned long long sum = (unsigned long long)g + (g | p);
        const uint32_t cin = (((uint32_t)sum ^ p) >> lane) & 1u;  // carry into this limb
        const bool over = (sum >> 32) != 0ull;                    // out of limb 31
        if (!over) X[pad(lane)] = (limb + cin) & LIMB_MASK;
        if (lane == 0) cs.flag = over ? 1u : 0u;
    }
    __syncthreads();
    if (cs.flag) {
        __syncthreads();
        while (c) c = carry_pass<true>(H, c, [&](int i) { return (unsigned long long)X[pad(i)]; }, X, cs);
    }
}

template <bool MUL, int LOGL>
__device__ void mont_step(const Smem &sm, const Cand &cd, bool square, uint32_t a, const Twiddles &tw,
                          const CrtConsts &cc, const uint32_t *gy = nullptr) {
    constexpr int L = 1 << LOGL, H = L >> 1, LOGH = LOGL - 1;
    constexpr int T = THREADS;
    constexpr bool FULL = LOGL <= LOG_LCTA;  // T from one length-L product
    uint32_t *A0 = sm.A0, *A1 = sm.A1, *X = sm.X;
    // the m and W products run on (P, Q); S waits in Sb until the end
    uint32_t *const P = FULL ? A0 : X, *const Q = A1, *const Sb = FULL ? X : A0;
    CarrySmem &cs = *sm.cs;
    const int tid = threadIdx.x;
    const bool prod = square || (MUL && gy);
    unsigned long long cS = 0;
    if constexpr (FULL) {
        if (prod) {
            // the first forward pass reads the H limbs from X itself
            if (MUL && gy) product_from<true, 0, LOGL, 1, true, true>(A0, A1, tw, gy, gy + L, cc, X);
            else product_from<true, 0, LOGL, 0, false, true>(A0, A1, tw, nullptr, nullptr, cc, X);
            carry_pass<true>(L, 0ull, [&](int i) { return crt(A0[pad(i)], A1[pad(i)], LOGL, cc); }, A0, cs);
            cS = carry_pass<true>(H, 0ull,
                                  [&](int i) { return (unsigned long long)A0[pad(i)] + A0[pad(i + H)]; }, X, cs);
            for (int i = tid; i < H; i += T) {  // D = T_lo - T_hi, limbs in (-B, B)
                const uint32_t lo = A0[pad(i)], hi = A0[pad(i + H)];
                A0[pad(i)] = lo + P1 - hi;
                A1[pad(i)] = lo + P2 - hi;
            }
        } else {  // T = X: S = D = X
            for (int i = tid; i < H; i += T) {
                const uint32_t v = X[pad(i)];
                A0[pad(i)] = v;
                A1[pad(i)] = v;
            }
        }
        __syncthreads();
    } else {
        if (prod) {
            // S: cyclic product in A0 (prime 1) and A1 (prime 2), kept in A0
            for (int i = tid; i < H; i += T) {
                const uint32_t v = X[pad(i)];
                A0[pad(i)] = v;
                A1[pad(i)] = v;
            }
            __syncthreads();
            if (MUL && gy) product_from<true, 0, LOGH, 1, true>(A0, A1, tw, gy, gy + L, cc);
            else product_from<true, 0, LOGH, 0, false>(A0, A1, tw, nullptr, nullptr, cc);
            cS = carry_pass<true>(H, 0ull, [&](int i) { return crt(A0[pad(i)], A1[pad(i)], LOGH, cc); }, A0, cs);
            // D: negacyclic product in X itself (prime 1) and A1 (prime 2), carried into X
            for (int i = tid; i < H; i += T) A1[pad(i)] = X[pad(i)];
            __syncthreads();
            if (MUL && gy) product_from<true, 0, LOGH, 1, true, false, true>(X, A1, tw, gy + H, gy + L + H, cc);
            else product_from<true, 0, LOGH, 0, false, false, true>(X, A1, tw, nullptr, nullptr, cc);
            const unsigned long long cD = carry_pass<true>(H, 0ull, [&](int i) {
                return crt_signed(X[pad(i)], A1[pad(i)], LOGH, cc, i == 0 ? OFF_N0 : OFF_C);
            }, X, cs);
            // D == X - cD (mod B^H + 1): cD < 2^39 folded into limbs 0 and 1 (signed limbs, mod p)
            const uint32_t c0 = (uint32_t)cD & LIMB_MASK, c1 = (uint32_t)(cD >> LIMB_BITS);
            for (int i = tid; i < H; i += T) {
                const uint32_t v = X[pad(i)], c = i == 0 ? c0 : (i == 1 ? c1 : 0u);
                X[pad(i)] = v + P1 - c;
                A1[pad(i)] = v + P2 - c;
            }
        } else {  // T = X: S = D = X
            for (int i = tid; i < H; i += T) {
                const uint32_t v = X[pad(i)];
                A0[pad(i)] = v;
                A1[pad(i)] = v;
            }
        }
        __syncthreads();
    }
    // m = D N'' (mod B^H + 1): negacyclic product on (P, Q), carried into P
    product_from<true, 0, LOGH, 1, false, false, true>(P, Q, tw, cd.nn, cd.nn + H, cc);
    const unsigned long long cM = carry_pass<true>(H, 0ull, [&](int i) {
        return crt_signed(P[pad(i)], Q[pad(i)], LOGH, cc, i == 0 ? OFF_N0 : OFF_C);
    }, P, cs);
    // m = lo - cM, plus R' when lo < cM (lo: the H limbs in P); modulo
    // B^H - 1 that is lo - cM + 2 neg.  lo < cM < 2^44 needs limbs 2.. zero:
    // the fold records that, and only then is limb 0 corrected.
    {
        const uint32_t m0 = (uint32_t)cM & LIMB_MASK, m1 = (uint32_t)(cM >> LIMB_BITS);
        bool z = true;
        for (int i = tid; i < H; i += T) {
            const uint32_t v = P[pad(i)], c = i == 0 ? m0 : (i == 1 ? m1 : 0u);
            z = z && (i < 2 || v == 0u);
            P[pad(i)] = v + P1 - c;
            Q[pad(i)] = v + P2 - c;
        }
        if (__syncthreads_and(z)) {
            if (tid == 0) {
                const unsigned long long lo =
                    ((unsigned long long)(P[pad(1)] - P1 + m1) << LIMB_BITS) | (P[pad(0)] - P1 + m0);
                if (lo < cM) {
                    P[pad(0)] += 2u;
                    Q[pad(0)] += 2u;
                }
            }
            __syncthreads();
        }
    }
    // W = m N (mod B^H - 1) on (P, Q), then V = S + W into X; end-around carries
    product_from<true, 0, LOGH, 1, false>(P, Q, tw, cd.nh, cd.nh + H, cc);
    unsigned long long c = carry_pass<true>(H, cS, [&](int i) {
        return (unsigned long long)Sb[pad(i)] + crt_signed(P[pad(i)], Q[pad(i)], LOGH, cc, OFF_C);
    }, X, cs);
    if (c) end_around(X, c, H, cs);
    // V = B^H - 1 represents 0 (U = 0: T = 0)
    bool ones = true;
    for (int i = tid; i < H; i += T) ones = ones && (X[pad(i)] == LIMB_MASK);
    if (__syncthreads_and(ones)) {
        for (int i = tid; i < H; i += T) X[pad(i)] = 0u;
        __syncthreads();
    }
    // X = a U from V = 2U
    if (a & 1u) {
        for (int i = tid; i < H; i += T) {
            const uint32_t nx = X[pad(i + 1 < H ? i + 1 : 0)];
            A1[pad(i)] = (X[pad(i)] >> 1) | ((nx & 1u) << (LIMB_BITS - 1));
        }
        __syncthreads();
        if (a > 1u) {
            carry_pass<true>(H, 0ull, [&](int i) { return (unsigned long long)A1[pad(i)] * a; }, X, cs);
        } else {
            for (int i = tid; i < H; i += T) X[pad(i)] = A1[pad(i)];
            __syncthreads();
        }
    } else if (a > 2u) {
        carry_pass<true>(H, 0ull, [&](int i) { return (unsigned long long)X[pad(i)] * (a >> 1); }, X, cs);
    }
}

}  // namespace mr
}  // namespace pfb
