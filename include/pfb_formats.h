/*
 * Text formats of the reference's runs, so outputs diff against a reference
 * run line for line.
 *
 *   candidate file   whitespace-separated records "a b c k j", as the MR
 *                    bench driver reads them (bench_mr_gpu.cu:159-171;
 *                    the repository's candidatos.txt)
 *   phase-1 file     one line per survivor:
 *                    "a=%lld b=%lld c=%lld k=%d j=%d"       (master.c:519-521)
 *   phase-2 file     one line per hit: the same fields followed by
 *                    " PROBABLE_PRIME_BOTH" (result 2) or " PRIME" (result 3)
 *                    (master.c:549-558); other results write nothing.
 *
 * Paths are host files; `append` non-zero appends (the master keeps its files
 * open across batches).  Return values: a count >= 0, or PFB_E_ARG / -7
 * (PFB_E_IO) with pfb_last_error() describing the failure.
 */
#pragma once
#include <stdint.h>

#include "pfb_pipeline.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PFB_E_IO (-7) /* a file could not be opened, read or written */

typedef struct {
    long long a, b, c;
    int k, j;
} pfb_candidate_t;

/* Reads up to cap records into out (out may be NULL with cap 0 to count);
 * returns the number of records in the file.  Reading stops at the first
 * token that is not an integer, as the reference's `fin >> a >> ...` does. */
long long pfb_read_candidates(const char *path, pfb_candidate_t *out, long long cap);

/* Writes the n records (a,b,c,k,j) of recs as phase-1 survivor lines. */
long long pfb_write_phase1(const char *path, const pfb_phase2_record_t *recs, long long n, int append);

/* Writes the records with result 2 or 3 as phase-2 lines; returns the lines
 * written. */
long long pfb_write_phase2(const char *path, const pfb_phase2_record_t *recs, long long n, int append);

#ifdef __cplusplus
}
#endif
