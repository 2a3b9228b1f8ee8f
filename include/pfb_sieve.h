/*
 * Wide-grid Phase-1 sieve: C ABI of the B200 sieve engine.
 *
 * The reference's ABI (trial_div.h:26-29) hard-wires a 100 x 100 (k,j) grid
 * (sieve_table.h:15-17, KJ_WORDS = 313).  This header extends it to a square
 * grid of side K (1 <= K <= 9999), several (a,b,c) triples per call, a prime
 * list kept resident in device memory, caller-chosen streams and on-device
 * survivor compaction.  It has no counterpart file in the reference; each
 * entry point names the reference code whose job it takes over.
 *
 * Mask layout (one block per triple): bit q = (k-1)*K + (j-1), LSB-first in
 * little-endian uint32 words, 1 = eliminated (p | N or p | rev(N) for some
 * prime of the list).  A block is pfb_sieve_mask_bytes(K) bytes = 4 *
 * ceil(K*K/32); at K = 100 it is exactly the reference's uint32_t[313].
 *
 * Errors: every entry point returns 0 on success and a negative PFB_E* code
 * otherwise; pfb_last_error() gives a one-line description.  Nothing here
 * throws or aborts.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PFB_OK = 0,
    PFB_E_ARG = -2,      /* invalid argument (sizes, null pointers, K range) */
    PFB_E_CUDA = -1,     /* a CUDA runtime call failed (same code as trial_div_gpu) */
    PFB_E_NOMEM = -3,    /* device allocation failed */
    PFB_E_CAPACITY = -4, /* output buffer too small / table full */
    PFB_E_TIMEOUT = -5,  /* a bounded device wait ran out */
    PFB_E_STATE = -6     /* call not valid in the object's current state */
};

#define PFB_SIEVE_MAX_K 9999

/* Flags for pfb_sieve_run. */
#define PFB_SIEVE_OR         1u  /* OR into the mask's current content (else overwrite) */
#define PFB_SIEVE_MASK_HOST  2u  /* mask points to host memory (else device memory)    */

typedef struct pfb_sieve pfb_sieve_t;

/* Thread-local description of the last error of this library, or "". */
const char *pfb_last_error(void);

/* Bytes of one per-triple mask block: 4 * ceil(K*K/32). */
size_t pfb_sieve_mask_bytes(int K);

/*
 * Create a sieve context on `device`: copies the prime list (host memory,
 * n_primes odd primes below 2^32; 2 is accepted; entries < 2 are ignored) to
 * device memory once and splits it by size.  Replaces the per-call cudaMalloc
 * + 23 MB upload of trial_div.cu:211-224.
 */
int pfb_sieve_create(pfb_sieve_t **out, const uint32_t *primes, uint32_t n_primes,
                     int device);
void pfb_sieve_destroy(pfb_sieve_t *s);

/*
 * Sieve n_abc triples (abc = {a0,b0,c0, a1,b1,c1, ...}, each >= 0) on the
 * K x K grid into mask (n_abc consecutive blocks).  The work of
 * trial_div_kernel (trial_div.cu:82-159) and sieve_one_prime
 * (trial_div_cpu.c:32-102), for any K.  stream is a cudaStream_t (NULL = the
 * context's own stream).  With a device mask the call is asynchronous; with
 * PFB_SIEVE_MASK_HOST it copies in/out and synchronises.  A call with a
 * different K than the previous one first waits for `stream` (the context
 * re-splits its prime list).  The context's working buffers are reused by
 * every call: calls on one context must be issued on one stream (or from one
 * thread with the stream synchronised between them); use one context per
 * concurrent stream.
 */
int pfb_sieve_run(pfb_sieve_t *s, const long long *abc, int n_abc, int K,
                  uint8_t *mask, unsigned flags, void *stream);

/*
 * Survivor compaction (replaces the host loop of worker.c:45-54): from one
 * device mask block, writes the surviving (k,j) (bit = 0) in k-major order as
 * uint32 (k << 16 | j) to d_out (device, capacity cap) and their number to
 * *count (host).  Synchronises on the stream.  Returns PFB_E_CAPACITY, with
 * *count set, if cap is too small.  Shares the context's working buffers
 * with pfb_sieve_run (same stream rule).
 */
int pfb_sieve_survivors(pfb_sieve_t *s, const uint8_t *d_mask, int K,
                        uint32_t *d_out, uint32_t cap, uint32_t *count, void *stream);

/*
 * Stateless convenience (the shape sketched for trial_div_gpu_grid): host
 * primes, host mask, synchronous, on the current device.  Keeps one internal
 * context per device and uploads the given prime list into it on every call
 * (as trial_div_gpu does); callers that sieve many batches with one list
 * should hold a pfb_sieve_t instead.
 */
int trial_div_gpu_grid(const uint32_t *primes, uint32_t n_primes,
                       const long long *abc, int n_abc, int K, uint8_t *mask_out,
                       unsigned flags);

/*
 * Allocation-free variant of pfb_sieve_run for one triple.  No counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc (a process
 * whose device memory is reserved up front by another allocator, or a loop
 * that cannot take the device-wide synchronisation cudaFree implies).
 *   d_primes  device array of n_primes odd primes
 *   d_mask    device mask block of pfb_sieve_mask_bytes(K) bytes, written
 *             (or OR-ed with PFB_SIEVE_OR) asynchronously on `stream`
 * Limits: one triple per call, 1 <= K <= 9999 (PFB_E_CAPACITY otherwise).
 * Working memory is one fixed __device__ array of 361 688 bytes (0.36 MB)
 * inside the library, held by every GPU that loads it until the process
 * exits; nothing is allocated.  All calls share that array: calls that
 * overlap on the GPU (two streams, two host threads) race and must be
 * serialised by the caller.  The first call on a device looks up the array's
 * device address and sets the tile kernel's shared-memory limit, and keeps
 * both for the life of the process; make that first call before any stream
 * capture, and do not call this entry point on a device again after
 * cudaDeviceReset on it (the kept address belongs to the old context).
 * Unlike pfb_sieve_run, which rejects a list repeating small primes
 * (PFB_E_ARG), this call lists each small value once, so a list with repeats
 * gives the mask of the list without them; even values below 10 000 are
 * skipped (2 never divides the odd N and rev(N)).
 */
int pfb_sieve_run_noalloc(const uint32_t *d_primes, uint32_t n_primes, long long a, long long b,
                          long long c, int K, uint32_t *d_mask, unsigned flags, void *stream);

#ifdef __cplusplus
}
#endif
