/*
 * Phase-2 test of one (a,b,c,k,j): drop-in for the reference's
 * miller_rabin.h:1-25 (same mr_timing_t and signature; worker.c:84 calls it).
 *
 * N = 10^a - k*10^b - j*10^c - 1, rev(N) = 10^a - rev(k)*10^(a-b-lk)
 * - rev(j)*10^(a-c-lj) - 1 (miller_rabin.c:56-99).  Returns 0 when N is
 * composite (rev(N) not tested), 1 when N is a probable prime and rev(N)
 * composite, 2 when both are probable primes; -1 on bad arguments or a GPU
 * failure.  The reference calls GMP's mpz_probab_prime_p(x, 5), which in GMP
 * 6.2+ is the Baillie-PSW test; this one runs the same test on the GPU (the
 * strong test to base 2, then the strong Lucas test with Selfridge's
 * parameters: pfb_mr_bpsw), so the verdicts are the same.
 */
#pragma once

typedef struct {
    double build_n;    /* build N                       */
    double mr_n;       /* probable-prime rounds on N    */
    double build_revn; /* build rev(N) (0 if N composite) */
    double mr_revn;    /* probable-prime rounds on rev(N) */
} mr_timing_t;

#ifdef __cplusplus
extern "C" {
#endif

int miller_rabin_test(long long a, long long b, long long c, int k, int j,
                      mr_timing_t *timing /* optional, may be NULL */);

#ifdef __cplusplus
}
#endif
