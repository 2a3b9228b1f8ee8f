/*
 * Phase-1 trial-division sieve: drop-in C ABI.
 *
 * Identical declarations to the reference's trial_div.h:1-36, so master.c /
 * worker.c (worker.c:38) and tests/test_gpu.c link against this library
 * unchanged.  The 100 x 100 (k,j) grid and its 313-word mask come from
 * sieve_table.h:15-17 (KJ_BITS / KJ_WORDS).
 */
#pragma once
#include "prime_list.h"
#include <stdint.h>

#ifndef KJ_BITS
#define BITS_PER_WORD 32
#define KJ_BITS  10000                                            /* 100 * 100 */
#define KJ_WORDS ((KJ_BITS + BITS_PER_WORD - 1) / BITS_PER_WORD)  /* 313 */
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* trial_div.h:10-14: per-step durations in seconds. */
typedef struct {
    double upload;    /* host -> device copies (primes + bits) */
    double kernel;    /* sieve kernels                          */
    double download;  /* device -> host copy of the bits        */
} gpu_timing_t;

/*
 * trial_div.h:16-29 / trial_div.cu:191-260.  For every prime p in pl and every
 * (k,j) in [1,100]^2, sets bit (k-1)*100+(j-1) of sieve_bits when p divides
 * N = 10^a - k*10^b - j*10^c - 1 or rev(N).  Bits are OR-ed into the caller's
 * array (phase-0 bits survive).  Synchronous on the current device.
 * Returns 0 on success, -1 on any CUDA error (one line on stderr).
 */
int trial_div_gpu(const prime_list_t *pl,
                  long long a, long long b, long long c,
                  uint32_t *sieve_bits /* KJ_WORDS uint32_t, in/out */,
                  gpu_timing_t *timing /* optional, may be NULL */);

/* trial_div.h:31-32 / trial_div.cu:173-181. */
int cuda_get_device_count(void);
int cuda_set_device(int index);  /* returns 0 on success */

#ifdef __cplusplus
}

/*
 * trial_div.cu:163-169 (C++ linkage, used by tests/bench_gpu.cu:25-27):
 * device pointers, asynchronous on the legacy default stream, 100 x 100 grid,
 * d_bits OR-ed.  block_size is accepted for source compatibility; the launch
 * shape is chosen by the library.
 */
void trial_div_launch(const uint32_t *d_primes, uint32_t n_primes,
                      uint64_t a, uint64_t b, uint64_t c,
                      uint32_t *d_bits, int block_size);
#endif
