// Host construction of the Miller-Rabin engine's constant tables: NTT
// twiddles with their Shoup companions, the CRT constants per transform
// length, and the twiddles of every radix-16 pass regrouped per group
// (WideTabs).  The engine uploads them once (build_tables in mr.cu); they
// are plain host computations so that the same tables can be built where no
// GPU is present.
#pragma once
#include <stdint.h>

#include <vector>

#include "mr_device.cuh"

namespace pfb {
namespace mr {

inline uint32_t powmod_h(uint64_t b, uint64_t e, uint32_t p) {
    uint64_t r = 1;
    b %= p;
    while (e) {
        if (e & 1) r = r * b % p;
        b = b * b % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

// floor(w 2^32 / p): the Shoup companion of w.
inline uint32_t shoup_c(uint32_t w, uint32_t p) { return (uint32_t)(((uint64_t)w << 32) / p); }

// 8 planes of 2^(LOG_LMAX-1) words: per prime p (p1 then p2) omega^k, its
// companion, omega^-k, its companion, omega of order 2^LOG_LMAX (3 is a
// primitive root of both primes).
inline std::vector<uint32_t> twiddle_table() {
    const int half = 1 << (LOG_LMAX - 1);
    std::vector<uint32_t> h((size_t)8 * half);
    const uint32_t P[2] = {P1, P2};
    for (int pr = 0; pr < 2; pr++) {
        const uint32_t p = P[pr];
        const uint32_t om = powmod_h(3, (p - 1) >> LOG_LMAX, p);
        const uint32_t omi = powmod_h(om, p - 2, p);
        uint32_t *w = h.data() + (size_t)(4 * pr + 0) * half, *wsh = w + half, *wi = wsh + half, *wish = wi + half;
        uint64_t a = 1, b = 1;
        for (int k = 0; k < half; k++) {
            w[k] = (uint32_t)a;
            wsh[k] = shoup_c((uint32_t)a, p);
            wi[k] = (uint32_t)b;
            wish[k] = shoup_c((uint32_t)b, p);
            a = a * om % p;
            b = b * omi % p;
        }
    }
    return h;
}

inline CrtConsts crt_consts() {
    const uint32_t P[2] = {P1, P2};
    CrtConsts cc{};
    const uint32_t ip1 = powmod_h(P1 % P2, P2 - 2, P2);
    const uint32_t two32_1 = (uint32_t)((1ull << 32) % P1), two32_2 = (uint32_t)((1ull << 32) % P2);
    for (int lg = 0; lg <= LOG_LMAX; lg++) {
        const uint32_t s1 = (uint32_t)((uint64_t)two32_1 * powmod_h(1ull << lg, P1 - 2, P1) % P1);
        const uint32_t s2 = (uint32_t)((uint64_t)two32_2 * powmod_h(1ull << lg, P2 - 2, P2) % P2);
        cc.s1[lg] = s1;
        cc.s1sh[lg] = shoup_c(s1, P1);
        cc.k2[lg] = (uint32_t)((uint64_t)s2 * ip1 % P2);
        cc.k2sh[lg] = shoup_c(cc.k2[lg], P2);
    }
    cc.k1 = ip1;
    cc.k1sh = shoup_c(ip1, P2);
    for (int pr = 0; pr < 2; pr++) {
        uint32_t inv = 1;  // p^-1 mod 2^32 by Newton
        for (int i = 0; i < 5; i++) inv *= 2u - P[pr] * inv;
        cc.pinv[pr] = 0u - inv;
    }
    return cc;
}

// Radix-16 pass tables (WideTabs): the twiddles load_tw would read, regrouped
// per j0, for every first-stage half size h0 a pass can have.  Returns the
// uint4 planes as words and fills wt.off (wt.base is left to the caller).
inline std::vector<uint32_t> wide_tables(const std::vector<uint32_t> &h, WideTabs &wt) {
    const int half = 1 << (LOG_LMAX - 1);
    std::vector<uint32_t> wide;  // as uint4 planes
    size_t off4 = 0;
    for (int dir = 0; dir < 2; dir++)
        for (int pr = 0; pr < 2; pr++) {
            const uint32_t *w = h.data() + (size_t)(4 * pr + 2 * dir) * half, *wsh = w + half;
            // forward passes: h0 = 8 .. 2^(LOG_LMAX-1), groups j0 < h0/8, element step h0/8;
            // inverse passes: h0 = 1 .. 2^(LOG_LMAX-4), groups j0 < h0, element step h0
            const int lmin = dir ? 0 : 3, lmax = dir ? LOG_LMAX - 4 : LOG_LMAX - 1;
            for (int lh0 = lmin; lh0 <= lmax; lh0++) {
                const int ng = dir ? (1 << lh0) : (1 << (lh0 - 3));
                const int step = ng;
                wt.off[dir][pr][lh0] = (uint32_t)off4;
                wide.resize((off4 + (size_t)8 * ng) * 4, 0u);
                for (int j0 = 0; j0 < ng; j0++) {
                    int t = 0;
                    for (int st = 0; st < 4; st++) {
                        const int cnt = dir ? (1 << st) : (16 >> (st + 1));
                        const int shift = dir ? LOG_LMAX - 1 - (lh0 + st) : LOG_LMAX - 1 - (lh0 - st);
                        for (int e = 0; e < cnt; e++, t++) {
                            const int k = (j0 + e * step) << shift;
                            const size_t plane = (size_t)(t >> 2), lane = (size_t)(t & 3);
                            wide[((off4 + plane * ng + j0) * 4) + lane] = w[k];
                            wide[((off4 + (4 + plane) * ng + j0) * 4) + lane] = wsh[k];
                        }
                    }
                }
                off4 += (size_t)8 * ng;
            }
        }
    return wide;
}

}  // namespace mr
}  // namespace pfb
