// Host side of the strong Lucas test: Selfridge's parameters for a modulus
// (the choice GMP's mpz_stronglucas makes inside mpz_probab_prime_p, which
// the reference's miller_rabin_test calls, miller_rabin.c:95,107).
#pragma once
#include <stdint.h>

#include <utility>

#include "bigint_host.h"

namespace pfb {
namespace mr {

inline uint32_t gcd_u32(uint32_t a, uint32_t b) {
    while (b) {
        const uint32_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// Jacobi symbol (a / n), n odd > 0.
inline int jacobi_u32(uint32_t a, uint32_t n) {
    a %= n;
    int t = 1;
    while (a) {
        while (!(a & 1u)) {
            a >>= 1;
            const uint32_t r = n & 7u;
            if (r == 3u || r == 5u) t = -t;
        }
        std::swap(a, n);
        if ((a & 3u) == 3u && (n & 3u) == 3u) t = -t;
        a %= n;
    }
    return n == 1u ? t : 0;
}

// Selfridge's method A for odd N > 1: D the first of 5, -7, 9, -11, ... with
// (D / N) = -1; Q = (1 - D) / 4.  Returns 1 with D set, 0 when N is composite
// (a factor gcd(|D|, N) < N, or a perfect square), -1 when no D with |D| <=
// 2001 works (not reached by non-squares in practice).
inline int selfridge(const pfb::big::Words &N, long &D_out) {
    using namespace pfb::big;
    const bool small = bit_length(N) <= 32;
    const int n_mod4 = (int)(N[0] & 3ull);
    long D = 5;
    for (int tries = 1;; tries++) {
        const uint32_t ad = (uint32_t)(D < 0 ? -D : D);
        const uint32_t r = mod_small(N, ad);
        const uint32_t g = gcd_u32(ad, r);
        if (g > 1u && !(small && N[0] == g)) return 0;
        // (|D| / N) = (N mod |D| / |D|) (-1)^((|D|-1)/2 (N-1)/2); (-1 / N) = (-1)^((N-1)/2)
        int j = jacobi_u32(r, ad);
        if ((ad & 3u) == 3u && n_mod4 == 3) j = -j;
        if (D < 0 && n_mod4 == 3) j = -j;
        if (j == -1) {
            D_out = D;
            return 1;
        }
        if (tries == 6) {  // (D / N) = -1 never happens for a square N
            const Words r2 = isqrt(N);
            if (cmp(mul(r2, r2), N) == 0) return 0;
        }
        D = D > 0 ? -(D + 2) : -D + 2;
        if ((D < 0 ? -D : D) > 2001) return -1;
    }
}

}  // namespace mr
}  // namespace pfb
