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
/* Device the engine was created on, or -1 for NULL. */
int pfb_mr_device(const pfb_mr_t *e);

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
 * Strong Lucas probable-prime test with Selfridge's parameters (method A: D
 * the first of 5, -7, 9, -11, ... with Jacobi (D/N) = -1, P = 1,
 * Q = (1 - D)/4): the second half of the Baillie-PSW test that GMP's
 * mpz_probab_prime_p runs for the reference's miller_rabin_test
 * (miller_rabin.c:95,107).  With N + 1 = 2^s d (d odd), N passes when
 * U_d == 0 or V_(d 2^r) == 0 (mod N) for some r < s.  verdict[i]: 1 strong
 * Lucas probable prime, 0 composite (a perfect square, or gcd(|D|, N) a proper
 * factor), -1 invalid (even, below 3, or too long for the ladder's headroom).
 */
int pfb_mr_lucas(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, int8_t *verdict);

/*
 * Baillie-PSW: the strong test to base 2, then pfb_mr_lucas on the numbers
 * that pass -- the decision GMP 6.2+ makes in mpz_probab_prime_p(N, reps) for
 * reps <= 24 (the reference calls it with reps = 5).  verdict[i]: 1 probable
 * prime, 0 composite (also even N > 2 and N < 2), -1 too long.
 */
int pfb_mr_bpsw(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, int8_t *verdict);

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
 *   advance  enqueue about `steps` steps of every unfinished candidate on
 *            `stream` (NULL = engine stream): a persistent kernel, one CTA
 *            per SM, hands out quanta of 64 steps round-robin, so the SMs
 *            stay busy whatever the number and lengths of the candidates
 *   pending  number of unfinished candidates (synchronises the device)
 *   results  verdicts / residues as in pfb_mr_test; PFB_E_STATE while some
 *            candidate is unfinished (its verdict is reported as -2)
 */
typedef struct pfb_mr_batch pfb_mr_batch_t;
int pfb_mr_batch_create(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base,
                        pfb_mr_batch_t **out);
int pfb_mr_batch_advance(pfb_mr_batch_t *b, int steps, void *stream);
int pfb_mr_batch_pending(pfb_mr_batch_t *b, int *pending);
/* Steps (squarings + checks) executed so far over all candidates (synchronises). */
long long pfb_mr_batch_steps_done(pfb_mr_batch_t *b);
long long pfb_mr_batch_steps_left(pfb_mr_batch_t *b);
int pfb_mr_batch_results(pfb_mr_batch_t *b, int8_t *verdict, uint16_t *residue, int residue_stride);
void pfb_mr_batch_destroy(pfb_mr_batch_t *b);

/*
 * Per-operation modular context: the reference's BatchModCtx methods
 * (batch_mod_ctx.cuh:132-179, batch_mod_ctx.cu:82-335) as a C ABI, run by
 * the engine one Montgomery step per call.  Operands use the reference's
 * layout: n_limbs 16-bit limbs per modulus, one per uint64, little-endian,
 * n_batch moduli back to back.  The working form ("residue") of x is
 * x R mod N, fully reduced, with R = 2^(22 H) of the modulus' transform
 * length H (the reference's Montgomery form with its own R).
 *   create        host set-up of every modulus (odd, > 1, at most
 *                 PFB_MR_MAX_BITS bits; PFB_E_ARG otherwise) and transforms
 *                 of N, N' (synchronous)
 *   to_residue    host x -> host working form (mod_residue_forward)
 *   from_residue  device working form -> host x (mod_residue_backward);
 *                 synchronises
 *   check_passed  d_passed[b] = (r_b is the working form of 1 or N - 1)
 *   modsq/modmul  d_out = working form of a^2 / a b, from working forms
 *   sq_raw/mul_raw  d_out = the full product, n_sum = 2 n_limbs + 16 limbs
 *                 per modulus (the reference's n_sum), no reduction
 * Device pointers; each call is asynchronous on `stream` (NULL = the legacy
 * default stream, where the reference's methods run, so that the caller's
 * cudaMemcpy calls are ordered with them); from_residue runs on the default
 * stream and returns when its result is on the host.  A context's scratch is
 * shared by its calls: calls on one context must not overlap on the GPU.
 */
typedef struct pfb_mr_ctx pfb_mr_ctx_t;
int pfb_mr_ctx_create(pfb_mr_t *e, const uint64_t *N_all, int n_limbs, int n_batch, pfb_mr_ctx_t **out);
void pfb_mr_ctx_destroy(pfb_mr_ctx_t *c);
int pfb_mr_ctx_n_sum(const pfb_mr_ctx_t *c);
/* Device arrays the context owns ([n_batch][n_limbs] 16-bit limbs in uint64):
 * the moduli, and the working forms of 1 and of N - 1.  Any may be NULL. */
int pfb_mr_ctx_buffers(const pfb_mr_ctx_t *c, const uint64_t **d_N, const uint64_t **d_one,
                       const uint64_t **d_nm1);
int pfb_mr_ctx_to_residue(pfb_mr_ctx_t *c, const uint64_t *x_all, uint64_t *out_all);
int pfb_mr_ctx_from_residue(pfb_mr_ctx_t *c, const uint64_t *d_x, uint64_t *out_all);
int pfb_mr_ctx_check_passed(pfb_mr_ctx_t *c, const uint64_t *d_r, uint8_t *d_passed, void *stream);
int pfb_mr_ctx_modsq(pfb_mr_ctx_t *c, const uint64_t *d_a, uint64_t *d_out, void *stream);
int pfb_mr_ctx_modmul(pfb_mr_ctx_t *c, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, void *stream);
int pfb_mr_ctx_sq_raw(pfb_mr_ctx_t *c, const uint64_t *d_a, uint64_t *d_out, void *stream);
int pfb_mr_ctx_mul_raw(pfb_mr_ctx_t *c, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, void *stream);

/*
 * Serving: continuous batching of strong tests (no counterpart in the
 * reference, which tests one fixed batch per call: bench_mr_gpu.cu:209-256).
 * Requests arrive one by one from any thread; host workers do the set-up;
 * a driver thread admits prepared requests into free device slots as slots
 * and the HBM budget allow, advances every resident candidate by
 * chunk_steps per launch of the persistent kernel (candidates of different
 * lengths share every launch), and retires finished ones.  Per-candidate
 * residue and exponent cursor live in device memory for the whole test.
 * If a slot allocation fails below the budget (device memory held
 * elsewhere), the server frees its pooled slot memory and retries; failing
 * that, the request waits until resident candidates retire, or gets verdict
 * -1 when none is resident.
 */
typedef struct pfb_mr_server pfb_mr_server_t;

typedef struct {
    int max_resident;          /* candidates on the GPU at once (0: 2 per SM)      */
    size_t hbm_budget_bytes;   /* cap on slot memory owned (0: no cap)             */
    int chunk_steps;           /* steps per candidate per launch (0: 512)          */
    uint32_t base;             /* witness, 2 <= base < 65536 (0: 2)                */
    int prep_threads;          /* host set-up threads (0: 4)                       */
} pfb_mr_server_config_t;

typedef struct {
    uint64_t tag;              /* caller's tag from pfb_mr_server_submit           */
    int8_t verdict;            /* 1 probable prime, 0 composite, -1 invalid input  */
    double submit_s, admit_s, done_s;  /* seconds since the server started         */
} pfb_mr_result_t;

typedef struct {
    long long submitted, admitted, completed, launches, steps_retired;
    int resident, queued, error;
    size_t bytes_in_use, bytes_owned;
} pfb_mr_server_stats_t;

int pfb_mr_server_create(pfb_mr_t *e, const pfb_mr_server_config_t *cfg, pfb_mr_server_t **out);
/* Queue N (16-bit limbs, copied).  residue_out (optional, host, residue_cap
 * limbs) receives base^d mod N before the result is posted. */
int pfb_mr_server_submit(pfb_mr_server_t *s, const uint16_t *limbs, int n_limbs, uint64_t tag,
                         uint16_t *residue_out, int residue_cap);
/* Up to cap finished results, waiting at most timeout_ms; returns their
 * number, or a negative PFB_E* code if the server stopped on an error. */
int pfb_mr_server_poll(pfb_mr_server_t *s, pfb_mr_result_t *out, int cap, int timeout_ms);
int pfb_mr_server_stats(pfb_mr_server_t *s, pfb_mr_server_stats_t *st);
/* Test hook (host-side fault injection; nothing faults on the device): the
 * next n allocations of slot memory fail as if cudaMalloc had returned
 * cudaErrorMemoryAllocation, exercising the server's recovery (free the
 * pooled blocks and retry; then requeue the request while others are
 * resident, or fail it with verdict -1 when none is).  Returns the number of
 * injected failures consumed so far. */
int pfb_mr_server_inject_alloc_failures(pfb_mr_server_t *s, int n);
/* Stops the loop (pending requests are dropped) and frees everything. */
void pfb_mr_server_destroy(pfb_mr_server_t *s);

/* Squarings (plus the final conversion) a strong test of N costs: the unit of
 * the engine's throughput counters. */
long long pfb_mr_test_cost(const uint16_t *limbs, int n_limbs);

/* Sustained 32-bit integer multiply rate of the device (ops/s), for the
 * low-half and high-half forms: the roofline denominator of the squaring
 * kernel.  No counterpart in the reference (a measurement utility). */
int pfb_measure_int32_peak(int device, double *mul_lo_per_s, double *mul_hi_per_s);

/*
 * Measurement utility (no counterpart in the reference): one radix-16 pass of
 * the squaring kernel's transform -- the first forward pass of a 2^14-point
 * transform, both primes -- in two forms on `ctas` CTAs, each on its own
 * 2^14 random limbs: the engine's butterfly pass (integer pipe) and an exact
 * int8 byte-plane matrix product on the tensor cores (tcgen05.mma kind::i8)
 * with the recombination on the CUDA cores.  Writes the mean time of one
 * launch of each form over `reps` launches, the number of output words on
 * which the two forms differ, and the tensor form's wait-timeout flag.
 */
int pfb_mr_radix16_forms(pfb_mr_t *e, int ctas, int reps, double *ms_butterfly, double *ms_tensor,
                         long long *mismatches, int *tensor_error);

/*
 * Autotuner of the persistent squaring kernel, per transform-length bucket
 * (log2 L from logl_lo to logl_hi, within 8..15; a 50 000-digit modulus is
 * 14, 100 000 digits 15).  For each bucket it times 2048 squarings of
 * synthetic moduli of the bucket's largest size, in batches of one and of two
 * candidates per SM, for every pair (quantum: steps of one candidate per
 * scheduling quantum, 16 to 64; chunk: steps per launch, 1024 or 2048), and
 * keeps in the engine, for every later batch of that bucket, the pair with
 * the best sum over the two shapes of its rate relative to the shape's best.
 * results (optional, cap rows) receives one row per pair; *n_results the rows
 * written.  The defaults before tuning are quantum 64, chunk 2048.
 */
typedef struct {
    int logl, quantum, chunk;
    double squarings_per_s_1;   /* whole device, one candidate per SM  */
    double squarings_per_s_2;   /* whole device, two candidates per SM */
} pfb_mr_tune_t;
int pfb_mr_autotune(pfb_mr_t *e, int logl_lo, int logl_hi, pfb_mr_tune_t *results, int cap,
                    int *n_results);
/* The (quantum, chunk) pair the engine uses for transform length 2^logl. */
int pfb_mr_get_tuning(pfb_mr_t *e, int logl, int *quantum, int *chunk);

#ifdef __cplusplus
}
#endif
