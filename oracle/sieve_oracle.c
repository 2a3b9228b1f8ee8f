/*
 * CPU oracle for the Phase-1 trial-division sieve (TEST INFRASTRUCTURE ONLY).
 *
 * This file is the checker for the CUDA sieve; nothing in the product links
 * it.  It restates the reference's CPU sieve (trial_div_cpu.c) for a square
 * grid of side K (1 <= K <= 9999) instead of the hard-wired 100 x 100 grid,
 * and adds the definitional brute force of tests/test_gpu.c.
 *
 *   N(k,j)    = 10^a - k*10^b - j*10^c - 1
 *   rev(N)    = 10^a - rev(k)*10^(a-b-lk) - rev(j)*10^(a-c-lj) - 1
 *               (miller_rabin.c:73-99; lk, lj = decimal digit counts)
 *
 * Mask layout: bit q = (k-1)*K + (j-1), LSB-first inside each byte,
 * 1 = eliminated.  At K = 100 this is byte-identical to the reference's
 * uint32_t sieve_bits[313] on a little-endian host.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* powmod_c, trial_div_cpu.c:22-30: square-and-multiply with 64-bit '%'. */
static uint64_t o_powmod(uint64_t base, uint64_t exp, uint32_t mod)
{
    uint64_t r = 1;
    base %= mod;
    while (exp > 0) {
        if (exp & 1) r = r * base % mod;
        base = base * base % mod;
        exp >>= 1;
    }
    return r % mod;
}

/* ndigits / rev_digits, miller_rabin.c:37-54, extended to 4 digits. */
static int o_ndig(int x) { return x < 10 ? 1 : x < 100 ? 2 : x < 1000 ? 3 : 4; }
static int o_rev(int x, int lx)
{
    int r = 0;
    for (int i = 0; i < lx; i++) { r = r * 10 + x % 10; x /= 10; }
    return r;
}

static inline void o_mark(uint8_t *mask, int K, int k, int j)
{
    uint64_t q = (uint64_t)(k - 1) * (uint64_t)K + (uint64_t)(j - 1);
    mask[q >> 3] |= (uint8_t)(1u << (q & 7));
}

/*
 * sieve_one_prime, trial_div_cpu.c:32-102, generalised from K = 100 to K.
 *  - normal form: j0 = (ra - k*rb - 1) * rc^-1, all j = j0 (mod p) in [1,K]
 *    (trial_div_cpu.c:40-52; skipped when rc == 0).
 *  - rev form, per k: base_k = ra - rev(k)*rb_rev[lk] - 1 (skipped when
 *    rb_rev[lk] == 0, :65-70); per digit class lj of j, rev(j) = base_k *
 *    rc_rev[lj]^-1 (mod p) (skipped when rc_rev[lj] == 0, :72-101).  The
 *    reference's lj = 2 branch (:82-95) maps rev values 1..9 to j = 10*rj and
 *    drops rev values ending in 0; the general rule below (j = rev_lj(rj),
 *    valid iff rj has no trailing zero, j <= K) reproduces it, and at K = 100
 *    the lj = 3 class holds only j = 100 (rj = 1), as at :97-100.
 *  - inverses by Fermat, powmod(x, p-2, p), as the reference does.
 */
static void o_sieve_one_prime(uint32_t p, long long a, long long b, long long c,
                              int K, uint8_t *mask)
{
    if (p < 2) return;
    uint64_t ra = o_powmod(10, (uint64_t)a, p);
    uint64_t rb = o_powmod(10, (uint64_t)b, p);
    uint64_t rc = o_powmod(10, (uint64_t)c, p);

    if (rc != 0) {
        uint64_t inv_rc = o_powmod(rc, (uint64_t)p - 2, p);
        for (int k = 1; k <= K; k++) {
            uint64_t num = (ra + 2 * (uint64_t)p - (uint64_t)k * rb % p - 1) % p;
            uint64_t j0 = num * inv_rc % p;
            if (j0 == 0) j0 = p;
            for (uint64_t j = j0; j <= (uint64_t)K; j += p) o_mark(mask, K, k, (int)j);
        }
    }

    int maxd = o_ndig(K);
    uint64_t rb_rev[5], rc_rev[5], inv_rev[5];
    for (int l = 1; l <= 4; l++) {
        long long eb = a - b - l, ec = a - c - l;
        rb_rev[l] = (eb >= 0) ? o_powmod(10, (uint64_t)eb, p) : 0;
        rc_rev[l] = (ec >= 0) ? o_powmod(10, (uint64_t)ec, p) : 0;
        inv_rev[l] = (rc_rev[l] != 0) ? o_powmod(rc_rev[l], (uint64_t)p - 2, p) : 0;
    }
    for (int k = 1; k <= K; k++) {
        int lk = o_ndig(k);
        uint64_t rk = (uint64_t)o_rev(k, lk);
        uint64_t rb_eff = rb_rev[lk];
        if (rb_eff == 0) continue;
        uint64_t base_k = (ra + 2 * (uint64_t)p - rk * rb_eff % p - 1) % p;
        for (int lj = 1; lj <= maxd; lj++) {
            if (inv_rev[lj] == 0) continue;
            uint64_t lim = (lj == 1) ? 9 : (lj == 2) ? 99 : (lj == 3) ? 999 : 9999;
            uint64_t trj = base_k * inv_rev[lj] % p;
            if (trj == 0) trj = p;
            for (uint64_t rj = trj; rj <= lim; rj += p) {
                if (lj > 1 && rj % 10 == 0) continue;   /* j would have fewer digits */
                int j = o_rev((int)rj, lj);
                if (j >= 1 && j <= K) o_mark(mask, K, k, j);
            }
        }
    }
}

/*
 * Restated trial_div_cpu() (trial_div_cpu.c:104-111) on a K x K grid, OR-ing
 * into mask.  The reference runs one prime after another on one thread; this
 * restatement splits the prime list over nthreads OpenMP threads, each with a
 * private mask, and ORs them (the result is order-independent).
 */
void oracle_sieve_grid(const uint32_t *primes, uint32_t n, long long a, long long b,
                       long long c, int K, uint8_t *mask, int nthreads)
{
    size_t nbytes = ((size_t)K * (size_t)K + 7) / 8;
    if (nthreads < 1) nthreads = 1;
#ifdef _OPENMP
    if (nthreads > 1) {
        uint8_t *priv = (uint8_t *)calloc((size_t)nthreads, nbytes);
        #pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4096)
        for (long long i = 0; i < (long long)n; i++) {
            int t = omp_get_thread_num();
            o_sieve_one_prime(primes[i], a, b, c, K, priv + (size_t)t * nbytes);
        }
        for (int t = 0; t < nthreads; t++) {
            const uint8_t *src = priv + (size_t)t * nbytes;
            for (size_t w = 0; w < nbytes; w++) mask[w] |= src[w];
        }
        free(priv);
        return;
    }
#endif
    for (uint32_t i = 0; i < n; i++) o_sieve_one_prime(primes[i], a, b, c, K, mask);
}

/*
 * Definitional brute force (tests/test_gpu.c:31-73): for every (k,j) and every
 * prime, evaluate N and rev(N) modulo p directly.  The rev residue uses the
 * reference's skip rules (a class whose power is 0 mod p, or whose exponent is
 * negative, eliminates nothing), so that it defines the same set as
 * trial_div_cpu.c for every p, including p = 5.  O(n * K^2): tiny inputs only.
 */
void oracle_sieve_brute(const uint32_t *primes, uint32_t n, long long a, long long b,
                        long long c, int K, uint8_t *mask)
{
    for (uint32_t i = 0; i < n; i++) {
        uint32_t p = primes[i];
        if (p < 2) continue;
        uint64_t ra = o_powmod(10, (uint64_t)a, p);
        uint64_t rb = o_powmod(10, (uint64_t)b, p);
        uint64_t rc = o_powmod(10, (uint64_t)c, p);
        uint64_t rbr[5], rcr[5];
        for (int l = 1; l <= 4; l++) {
            long long eb = a - b - l, ec = a - c - l;
            rbr[l] = (eb >= 0) ? o_powmod(10, (uint64_t)eb, p) : 0;
            rcr[l] = (ec >= 0) ? o_powmod(10, (uint64_t)ec, p) : 0;
        }
        for (int k = 1; k <= K; k++) {
            int lk = o_ndig(k);
            uint64_t rk = (uint64_t)o_rev(k, lk);
            for (int j = 1; j <= K; j++) {
                int lj = o_ndig(j);
                uint64_t rj = (uint64_t)o_rev(j, lj);
                int hit = 0;
                if (rc != 0) {
                    uint64_t v = (ra + 3 * (uint64_t)p - (uint64_t)k % p * rb % p
                                  - (uint64_t)j % p * rc % p - 1) % p;
                    hit = (v == 0);
                }
                if (!hit && rbr[lk] != 0 && rcr[lj] != 0) {
                    uint64_t v = (ra + 3 * (uint64_t)p - rk % p * rbr[lk] % p
                                  - rj % p * rcr[lj] % p - 1) % p;
                    hit = (v == 0);
                }
                if (hit) o_mark(mask, K, k, j);
            }
        }
    }
}

/* Decimal digit reversal helpers, exported for the host-side tests. */
int oracle_ndigits(int x) { return o_ndig(x); }
int oracle_rev_digits(int x, int lx) { return o_rev(x, lx); }

/*
 * Gap-coded prime file writer and reader: the format of gen_primes.c:1-11
 * and prime_list.c:5-55 ([u32 count][u32 first][u8 gap...], gap 0 escapes
 * to a little-endian u16).  Used to produce the prime list on the fly.
 */
uint32_t oracle_primes_below(uint32_t limit, uint32_t *out, uint32_t cap)
{
    /* plain odd-only Eratosthenes; 2 is excluded like gen_primes.c:119-122 */
    if (limit < 4) return 0;
    uint32_t half = (limit - 1) / 2;                 /* odd numbers 3..limit */
    uint8_t *comp = (uint8_t *)calloc(half + 1, 1);
    for (uint64_t i = 1; (2 * i + 1) * (2 * i + 1) <= limit; i++) {
        if (comp[i]) continue;
        uint64_t p = 2 * i + 1;
        for (uint64_t m = p * p; m <= limit; m += 2 * p) comp[(m - 1) / 2] = 1;
    }
    uint32_t cnt = 0;
    for (uint64_t i = 1; i <= half; i++) {
        uint64_t v = 2 * i + 1;
        if (v > limit) break;
        if (!comp[i]) {
            if (out && cnt < cap) out[cnt] = (uint32_t)v;
            cnt++;
        }
    }
    free(comp);
    return cnt;
}
