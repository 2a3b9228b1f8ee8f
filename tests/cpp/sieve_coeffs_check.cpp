// The line coefficients of the large-prime kernels (line_coeffs_m: Montgomery
// products, shared squaring chains) against the small-prime set-up's
// (line_coeffs: Barrett powers) and against plain 128-bit powers, for primes
// from 7 to just below 2^32 and triples with exponents of either sign.
// Prints "ok <cases>" or the first mismatch.
#include <cstdio>
#include <random>
#include <vector>

#include "sieve_device.cuh"

static bool is_prime(uint32_t n) {
    if (n < 2) return false;
    for (uint64_t d = 2; d * d <= n; d++)
        if (n % d == 0) return false;
    return true;
}

static uint32_t pw(uint32_t p, long long e) {  // 10^e mod p for any integer e, p prime, p != 2, 5
    unsigned long long base = 10 % p, ex = e >= 0 ? (unsigned long long)e : (unsigned long long)(-e);
    if (e < 0) {  // 10^-1 = 10^(p-2)
        unsigned long long r = 1, b = base, k = p - 2;
        while (k) {
            if (k & 1) r = (unsigned __int128)r * b % p;
            b = (unsigned __int128)b * b % p;
            k >>= 1;
        }
        base = r;
    }
    unsigned long long r = 1 % p;
    while (ex) {
        if (ex & 1) r = (unsigned __int128)r * base % p;
        base = (unsigned __int128)base * base % p;
        ex >>= 1;
    }
    return (uint32_t)r;
}

int main() {
    std::mt19937_64 rng(11);
    std::vector<uint32_t> primes;
    const uint64_t bands[][2] = {{7, 100}, {10000, 20000}, {1u << 20, (1u << 20) + 5000}, {99990000, 100000000},
                                 {2147480000u, 2147483648u}, {4294960000u, 4294967295u}};
    for (auto &b : bands) {
        int got = 0;
        for (uint64_t n = b[1]; n > b[0] && got < 40; n--)
            if (n % 2 && n % 5 && is_prime((uint32_t)n)) {
                primes.push_back((uint32_t)n);
                got++;
            }
    }
    long long cases = 0;
    for (uint32_t p : primes)
        for (int it = 0; it < 30; it++) {
            const long long a = (long long)(rng() % 200000), b = (long long)(rng() % 200000),
                            c = (long long)(rng() % 200000);
            for (int D = 1; D <= 4; D++) {
                Mod32 B;
                B.init(p);
                LineCoeffs lb;
                line_coeffs(B, a, b, c, D, lb);
                Mont32 M;
                M.init(p);
                LineCoeffsM lm;
                line_coeffs_m(M, a, b, c, D, lm);
                const uint32_t ram1 = (uint32_t)(((unsigned long long)pw(p, a) + p - 1) % p);
                const uint32_t an = (uint32_t)((unsigned long long)ram1 * pw(p, -c) % p);
                const uint32_t ar = (uint32_t)((unsigned long long)ram1 * pw(p, c + D - a) % p);
                const uint32_t bn = pw(p, b - c), br = pw(p, c - b);
                const uint32_t R = (uint32_t)((1ull << 32) % p);
                const bool ok = lm.an == an && lm.bn == bn && lm.ar == ar && lm.br == br && lb.an == an &&
                                lb.bn == bn && lb.ar == ar && lb.br == br &&
                                lm.bnm == (uint32_t)((unsigned long long)bn * R % p) &&
                                lm.brm == (uint32_t)((unsigned long long)br * R % p);
                if (!ok) {
                    printf("mismatch p=%u a=%lld b=%lld c=%lld D=%d\n", p, a, b, c, D);
                    return 1;
                }
                cases++;
            }
        }
    printf("ok %lld\n", cases);
    return 0;
}
