/*
 * Phase-0 periodic sieve table on the GPU (the reference's sieve_table.c /
 * sieve.c, built on the CPU by its master at start-up: master.c:430-433).
 *
 * For a small prime p with L = ord_p(10), N mod p and rev(N) mod p depend on
 * (a, b, c) only through (a mod L, b mod L, c mod L).  The table holds, for
 * every prime p >= 3 of the given list with L defined and L^3 <= 2^18, the
 * 100 x 100 elimination mask (313 words, bit (k-1)*100 + (j-1)) of each
 * residue triple -- for the primes below 1e4, 62 primes and 3 208 136 masks,
 * 4.0 GB of device memory, filled by one kernel.  Applying it to (a, b, c)
 * ORs one mask per prime (sieve_apply, sieve.c:4-22).  The masks are those of
 * sieve_table.c:93-178 bit for bit, including its rev(N) exponents taken mod L
 * (so they are defined even where a - b - lk or a - c - lj is negative).
 *
 * Errors: 0 or a negative PFB_E* code (pfb_sieve.h), pfb_last_error().
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "pfb_sieve.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pfb_phase0 pfb_phase0_t;

/* Build the table on `device` from host primes (the reference uses the primes
 * below 1e4).  Synchronous. */
int pfb_phase0_create(pfb_phase0_t **out, const uint32_t *primes, uint32_t n_primes, int device);

/* Masks of n_abc triples (a, b, c >= 0): n_abc blocks of 313 words, written
 * or OR-ed (PFB_SIEVE_OR) into `masks`, device memory (asynchronous on
 * `stream`) or host memory (PFB_SIEVE_MASK_HOST, synchronous). */
int pfb_phase0_apply(pfb_phase0_t *t, const long long *abc, int n_abc, uint32_t *masks, unsigned flags,
                     void *stream);

/* Tabled primes, masks and device bytes of the table; seconds the build took. */
int pfb_phase0_info(pfb_phase0_t *t, int *n_primes, long long *n_masks, size_t *table_bytes,
                    double *build_seconds);

void pfb_phase0_destroy(pfb_phase0_t *t);

#ifdef __cplusplus
}
#endif
