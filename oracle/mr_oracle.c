/*
 * CPU oracle for the Miller-Rabin path (TEST INFRASTRUCTURE ONLY).
 *
 * Everything here runs GMP 6.3 (libgmp.so.10), the arithmetic the reference
 * trusts: miller_rabin.c:101-143 calls mpz_probab_prime_p(x, 5), and the
 * reference's GPU test-suite checks its NTT arithmetic against mpz_mul /
 * mpz_powm (miller_rabin_gpu/correctness_tests.cuh:252-746).  The product
 * never links this file.
 *
 * Numbers cross the boundary as little-endian 16-bit limbs (uint16_t), the
 * limb width of the reference's GPU path (ntt_merge.cuh:14-19,
 * candidate.cuh:11-18).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "gmp.h"

static void o_from_limbs(mpz_t x, const uint16_t *limbs, int n)
{
    mpz_import(x, (size_t)n, -1, sizeof(uint16_t), 0, 0, limbs);
}

static int o_to_limbs(const mpz_t x, uint16_t *out, int cap)
{
    size_t cnt = 0;
    int need = (int)((mpz_sizeinbase(x, 2) + 15) / 16);
    if (mpz_cmp_ui(x, 0) == 0) need = 0;
    if (need > cap) return -1;
    memset(out, 0, sizeof(uint16_t) * (size_t)cap);
    if (need) mpz_export(out, &cnt, -1, sizeof(uint16_t), 0, 0, x);
    return need;
}

/* ndigits / rev_digits of miller_rabin.c:37-54 (k, j up to 4 digits). */
static int o_ndig(int x) { return x < 10 ? 1 : x < 100 ? 2 : x < 1000 ? 3 : 4; }
static int o_rev(int x, int lx)
{
    int r = 0;
    for (int i = 0; i < lx; i++) { r = r * 10 + x % 10; x /= 10; }
    return r;
}

/*
 * build_N / build_revN, miller_rabin.c:56-99 (also candidate.cuh:77-98):
 *   N      = 10^a - k*10^b - j*10^c - 1
 *   rev(N) = 10^a - rev(k)*10^(a-b-lk) - rev(j)*10^(a-c-lj) - 1
 * Writes little-endian 16-bit limbs; returns the limb count or -1 if cap is
 * too small / an exponent is negative.
 */
int oracle_build_candidate(long long a, long long b, long long c, int k, int j,
                           int rev, uint16_t *out, int cap)
{
    mpz_t x, t;
    mpz_init(x);
    mpz_init(t);
    long long eb = b, ec = c;
    unsigned long mk = (unsigned long)k, mj = (unsigned long)j;
    if (rev) {
        int lk = o_ndig(k), lj = o_ndig(j);
        eb = a - b - lk;
        ec = a - c - lj;
        mk = (unsigned long)o_rev(k, lk);
        mj = (unsigned long)o_rev(j, lj);
    }
    if (a < 0 || eb < 0 || ec < 0) { mpz_clear(x); mpz_clear(t); return -1; }
    mpz_ui_pow_ui(x, 10, (unsigned long)a);
    mpz_ui_pow_ui(t, 10, (unsigned long)eb);
    mpz_mul_ui(t, t, mk);
    mpz_sub(x, x, t);
    mpz_ui_pow_ui(t, 10, (unsigned long)ec);
    mpz_mul_ui(t, t, mj);
    mpz_sub(x, x, t);
    mpz_sub_ui(x, x, 1);
    int r = (mpz_cmp_ui(x, 0) > 0) ? o_to_limbs(x, out, cap) : -1;
    mpz_clear(x);
    mpz_clear(t);
    return r;
}

/*
 * Strong-test residue: N - 1 = 2^s * d (d odd), r = base^d mod N
 * (mpz_powm).  Returns s (>= 1), or -1 for even/too-small N.  The residue
 * is written as n_out limbs.
 */
int oracle_strong_residue(const uint16_t *n_limbs, int n, unsigned long base,
                          uint16_t *res, int n_out)
{
    mpz_t N, d, g, r;
    mpz_init(N); mpz_init(d); mpz_init(g); mpz_init(r);
    o_from_limbs(N, n_limbs, n);
    int s = -1;
    if (mpz_cmp_ui(N, 3) >= 0 && mpz_odd_p(N)) {
        mpz_sub_ui(d, N, 1);
        s = (int)mpz_scan1(d, 0);
        mpz_tdiv_q_2exp(d, d, (mp_bitcnt_t)s);
        mpz_set_ui(g, base);
        mpz_powm(r, g, d, N);
        if (o_to_limbs(r, res, n_out) < 0) s = -1;
    }
    mpz_clear(N); mpz_clear(d); mpz_clear(g); mpz_clear(r);
    return s;
}

/*
 * Full strong probable-prime test to one base (the Miller-Rabin round the
 * reference's gpu_miller_rabin / gpu_miller_rabin_s1 run per witness,
 * miller_rabin_runner.cu:281-473): 1 if base^d == +-1 or base^(d*2^i) == -1
 * for some 0 < i < s, else 0.  -1 on bad input.
 */
int oracle_strong_test(const uint16_t *n_limbs, int n, unsigned long base)
{
    mpz_t N, d, g, r, nm1;
    mpz_init(N); mpz_init(d); mpz_init(g); mpz_init(r); mpz_init(nm1);
    o_from_limbs(N, n_limbs, n);
    int out = -1;
    if (mpz_cmp_ui(N, 3) >= 0 && mpz_odd_p(N)) {
        mpz_sub_ui(nm1, N, 1);
        int s = (int)mpz_scan1(nm1, 0);
        mpz_tdiv_q_2exp(d, nm1, (mp_bitcnt_t)s);
        mpz_set_ui(g, base);
        mpz_powm(r, g, d, N);
        out = 0;
        if (mpz_cmp_ui(r, 1) == 0 || mpz_cmp(r, nm1) == 0) out = 1;
        for (int i = 1; i < s && !out; i++) {
            mpz_mul(r, r, r);
            mpz_mod(r, r, N);
            if (mpz_cmp(r, nm1) == 0) out = 1;
        }
    }
    mpz_clear(N); mpz_clear(d); mpz_clear(g); mpz_clear(r); mpz_clear(nm1);
    return out;
}

/* mpz_probab_prime_p(N, reps): 0 composite, 1 probable prime, 2 prime. */
int oracle_probab_prime(const uint16_t *n_limbs, int n, int reps)
{
    mpz_t N;
    mpz_init(N);
    o_from_limbs(N, n_limbs, n);
    int r = mpz_probab_prime_p(N, reps);
    mpz_clear(N);
    return r;
}

/* Plain modular product and power, for arithmetic unit tests. */
int oracle_mulmod(const uint16_t *x, const uint16_t *y, const uint16_t *m, int n,
                  uint16_t *out)
{
    mpz_t X, Y, M;
    mpz_init(X); mpz_init(Y); mpz_init(M);
    o_from_limbs(X, x, n); o_from_limbs(Y, y, n); o_from_limbs(M, m, n);
    mpz_mul(X, X, Y);
    mpz_mod(X, X, M);
    int r = o_to_limbs(X, out, n);
    mpz_clear(X); mpz_clear(Y); mpz_clear(M);
    return r;
}

int oracle_powm(const uint16_t *base, int nb, const uint16_t *exp, int ne,
                const uint16_t *m, int n, uint16_t *out)
{
    mpz_t B, E, M, R;
    mpz_init(B); mpz_init(E); mpz_init(M); mpz_init(R);
    o_from_limbs(B, base, nb); o_from_limbs(E, exp, ne); o_from_limbs(M, m, n);
    mpz_powm(R, B, E, M);
    int r = o_to_limbs(R, out, n);
    mpz_clear(B); mpz_clear(E); mpz_clear(M); mpz_clear(R);
    return r;
}

/* Next prime above x (mpz_nextprime), used for the 2^512-seeded KATs. */
int oracle_nextprime(const uint16_t *x, int n, uint16_t *out, int cap)
{
    mpz_t X;
    mpz_init(X);
    o_from_limbs(X, x, n);
    mpz_nextprime(X, X);
    int r = o_to_limbs(X, out, cap);
    mpz_clear(X);
    return r;
}
