/*
 * Batched Miller-Rabin engine: C ABI.
 *
 * Takes over the job of the reference's GPU Miller-Rabin library
 * (miller_rabin_gpu/: BatchModCtx batch_mod_ctx.cuh:101-228,
 * gpu_miller_rabin_s1 / gpu_miller_rabin miller_rabin_runner.cuh:26-49) and
 * of the CPU phase-2 call miller_rabin_test (miller_rabin.h:24-25), with the
 * arithmetic on the GPU: exact NTT squaring over two 30-bit primes,
 * Montgomery reduction and carry propagation fused in one CTA per candidate.
 *
 * Numbers cross this boundary as little-endian 16-bit limbs, the limb format
 * of the reference (ntt_merge.cuh:14-19, candidate.cuh:11-18); candidates of
 * different lengths may share one call.  Limits: 3 <= N, N odd,
 * bits(N) <= PFB_MR_MAX_BITS; witness bases 2 <= a < 65536.
 *
 * Every entry point returns 0 (PFB_OK) or a negative PFB_E* code (see
 * pfb_sieve.h) and never throws; pfb_last_error() describes the failure.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "pfb_sieve.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Largest modulus: R = 2^(22*H), H = 2^14 limbs, minus a 36-bit margin
 * (108 495 decimal digits). */
#define PFB_MR_MAX_BITS (22 * 16384 - 36)

typedef struct pfb_mr pfb_mr_t;

typedef struct {
    const uint16_t *limbs;  /* little-endian 16-bit limbs */
    int n_limbs;
} pfb_mr_number_t;

/* Engine on `device`: twiddle tables and constants are set up once. */
int pfb_mr_create(pfb_mr_t **out, int device);
void pfb_mr_destroy(pfb_mr_t *e);

/*
 * Strong probable-prime test (one Miller-Rabin round) to base `base` for n
 * numbers, all resident on the GPU at once (the batched form of
 * gpu_miller_rabin_s1 / gpu_miller_rabin, miller_rabin_runner.cu:281-473).
 *   verdict[i] = 1  probable prime (a^d == +-1 or a^(d 2^r) == -1, r < s)
 *              = 0  composite
 *              = -1 invalid input (even, < 3, too long): no work done
 * residue (optional, n * residue_stride limbs): a^d mod N_i with
 * N_i - 1 = 2^s d, d odd, as 16-bit limbs (zero-filled), the value
 * mpz_powm(a, d, N) gives.  Synchronous.
 */
int pfb_mr_test(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base,
                int8_t *verdict, uint16_t *residue, int residue_stride);

/*
 * Modular power with a small base: residue_i = base^exp_i mod N_i (the
 * windowed exponentiation of window_exp_loop, miller_rabin_runner.cu:89-203,
 * for base < 2^16).  exp_i are 16-bit limbs (exp_limbs[i], n_exp[i] each) and
 * must be >= 1.  N_i odd.  Synchronous.
 */
int pfb_mr_powm(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base,
                const pfb_mr_number_t *exps, uint16_t *residue, int residue_stride);

/*
 * Resident batches: the same tests as pfb_mr_test, driven step by step (the
 * job of BatchModCtx + the witness loop, batch_mod_ctx.cuh:101-228 and
 * miller_rabin_runner.cu:281-359, with the candidates' state kept in device
 * memory between calls).  A step is one modular squaring of every unfinished
 * candidate (or one verdict check).
 *   create   host set-up, upload and transforms of N and N' (synchronous)
 *   advance  enqueue `steps` steps on `stream` (NULL = engine stream)
 *   pending  number of unfinished candidates (synchronises the device)
 *   results  verdicts / residues as in pfb_mr_test; PFB_E_STATE while some
 *            candidate is unfinished (its verdict is reported as -2)
 */
typedef struct pfb_mr_batch pfb_mr_batch_t;
int pfb_mr_batch_create(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base,
                        pfb_mr_batch_t **out);
int pfb_mr_batch_advance(pfb_mr_batch_t *b, int steps, void *stream);
int pfb_mr_batch_pending(pfb_mr_batch_t *b, int *pending);
long long pfb_mr_batch_steps_left(pfb_mr_batch_t *b);
int pfb_mr_batch_results(pfb_mr_batch_t *b, int8_t *verdict, uint16_t *residue, int residue_stride);
void pfb_mr_batch_destroy(pfb_mr_batch_t *b);

/* Squarings (plus the final conversion) a strong test of N costs: the unit of
 * the engine's throughput counters. */
long long pfb_mr_test_cost(const uint16_t *limbs, int n_limbs);

/* Sustained 32-bit integer multiply rate of the device (ops/s), for the
 * low-half and high-half forms: the roofline denominator of the squaring
 * kernel.  No counterpart in the reference (a measurement utility). */
int pfb_measure_int32_peak(int device, double *mul_lo_per_s, double *mul_hi_per_s);

#ifdef __cplusplus
}
#endif
