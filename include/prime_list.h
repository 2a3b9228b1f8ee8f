/*
 * prime_list_t — the prime list handed to the Phase-1 sieve.
 *
 * Same layout and entry points as the reference's prime_list.h:1-19
 * (prime_list.c:12-62 implements the loader for the gap-coded file written
 * by gen_primes.c).  Primes are odd, ascending, below 2^32.
 */
#pragma once
#include <stdint.h>

typedef struct {
    uint32_t *primes;
    uint32_t  count;
} prime_list_t;

#ifdef __cplusplus
extern "C" {
#endif

/* Load a gap-coded prime file: [u32 count][u32 first][u8 gap...], a gap of 0
 * escapes to a little-endian u16 (prime_list.c:5-55).  Returns 0 on success. */
int  prime_list_load(prime_list_t *pl, const char *path);
void prime_list_free(prime_list_t *pl);

/* Write the same gap-coded format (the file gen_primes.c:21-133 produces) from
 * an ascending array; gaps above 65535 are rejected.  Returns 0 on success. */
int  prime_list_save(const uint32_t *primes, uint32_t count, const char *path);

#ifdef __cplusplus
}
#endif
