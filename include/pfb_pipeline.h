/*
 * Phase 1 -> Phase 2 on one GPU: sieve a list of (a,b,c) triples on the
 * K x K grid, compact the survivors on the device, and decide every survivor
 * with the GPU probable-prime engine.
 *
 * Takes over the work the reference spreads over an MPI master and its
 * workers: do_gpu_task (worker.c:15-66: trial_div_gpu on a 313-word mask, then
 * a host scan of the survivors), the master's queue of Phase-2 tasks, and
 * do_cpu_task (worker.c:68-107: miller_rabin_test per surviving (k,j)).  Here
 * the survivors stay on the device until compacted (4 bytes each cross to the
 * host), N is built on the host from cached powers of ten, and the base-2
 * strong tests of all survivors run through one continuous-batching server
 * (pfb_mr_server_*), so the tests of one triple overlap the sieve and tests of
 * the others.
 *
 * Result codes per survivor are those of miller_rabin_test (miller_rabin.h,
 * messages.h:57-66): 0 N composite, 1 N probable prime and rev(N) composite,
 * 2 both probable primes; -1 when rev(N) cannot be formed (a negative
 * exponent a-b-lk or a-c-lj) or N < 1.  The probable-prime decision is the
 * one miller_rabin_test makes in this library.
 *
 * Errors: 0 on success, a negative PFB_E* code otherwise (pfb_last_error()).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "pfb_mr.h"
#include "pfb_sieve.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    long long a, b, c;   /* the triple                                  */
    int k, j;            /* surviving cell, 1-based                     */
    int result;          /* miller_rabin_test code (see above)          */
} pfb_phase2_record_t;

typedef struct {
    int K;                     /* grid side, 1 <= K <= 9999                         */
    int triples_per_sieve;     /* triples per sieve call (0: 8)                     */
    int max_resident;          /* candidates on the GPU at once (0: 2 per SM)       */
    size_t hbm_budget_bytes;   /* cap on the test server's slot memory (0: none)    */
    int prep_threads;          /* host set-up threads of the server (0: 4)          */
    int window;                /* survivors in flight in the server (0: 4 x slots)  */
} pfb_pipeline_config_t;

typedef struct {
    long long triples, survivors, n_prp, rev_tested, both_prp, invalid;
    double sieve_s, phase2_s, total_s;
} pfb_pipeline_stats_t;

/*
 * Run the pipeline over n_abc triples (abc = {a0,b0,c0, ...}).  pre_mask, if
 * not NULL, holds n_abc host mask blocks (pfb_sieve_mask_bytes(K) bytes each,
 * the layout of pfb_sieve.h) whose set bits are eliminated before sieving: the
 * Phase-0 bits of gpu_task_t.sieve_bits (messages.h:31-34).  Records are
 * written to out in triple order, k-major within a triple (worker.c:45-54).
 * If cap is smaller than the number of survivors, nothing is tested,
 * *n_out is set to that number and PFB_E_CAPACITY is returned.  sv and mr
 * must live on the same device; mr must not be used by another thread during
 * the call.
 */
int pfb_pipeline_run(pfb_sieve_t *sv, pfb_mr_t *mr, const long long *abc, int n_abc,
                     const pfb_pipeline_config_t *cfg, const uint8_t *pre_mask,
                     pfb_phase2_record_t *out, long long cap, long long *n_out,
                     pfb_pipeline_stats_t *stats);

#ifdef __cplusplus
}
#endif
