// Gap-coded prime files (host code).
//
// Reader with the behaviour of prime_list_load / prime_list_free
// (prime_list.c:12-62) and a writer for the format gen_primes.c:1-11 emits:
//   [u32 count][u32 first prime][u8 gap ...], gap 0 escapes to a
//   little-endian u16 gap.
// Written here so the library is self-contained for callers that do not link
// the reference's prime_list.c.
#include <stdio.h>
#include <stdlib.h>

#include "common.cuh"
#include "prime_list.h"

extern "C" int prime_list_load(prime_list_t *pl, const char *path) {
    if (!pl || !path) return -1;
    pl->primes = nullptr;
    pl->count = 0;
    FILE *f = fopen(path, "rb");
    if (!f) {
        perror(path);
        return -1;
    }
    uint32_t count = 0;
    if (fread(&count, sizeof(count), 1, f) != 1) {
        fclose(f);
        return -1;
    }
    uint32_t *p = (uint32_t *)malloc((size_t)(count ? count : 1) * sizeof(uint32_t));
    if (!p) {
        fclose(f);
        return -1;
    }
    bool ok = true;
    if (count) ok = fread(&p[0], sizeof(uint32_t), 1, f) == 1;
    for (uint32_t i = 1; ok && i < count; i++) {
        int g = fgetc(f);
        if (g == EOF) { ok = false; break; }
        uint32_t gap = (uint32_t)g;
        if (gap == 0) {
            int lo = fgetc(f), hi = fgetc(f);
            if (lo == EOF || hi == EOF) { ok = false; break; }
            gap = (uint32_t)lo | ((uint32_t)hi << 8);
        }
        p[i] = p[i - 1] + gap;
    }
    fclose(f);
    if (!ok) {
        free(p);
        return -1;
    }
    pl->primes = p;
    pl->count = count;
    return 0;
}

extern "C" void prime_list_free(prime_list_t *pl) {
    if (!pl) return;
    free(pl->primes);
    pl->primes = nullptr;
    pl->count = 0;
}

// Writer (no counterpart entry point in the reference: gen_primes.c writes
// the same format from its own sieve).  Primes must be ascending.
extern "C" int prime_list_save(const uint32_t *primes, uint32_t count, const char *path) {
    if ((count && !primes) || !path) return -1;
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    bool ok = fwrite(&count, sizeof(count), 1, f) == 1;
    if (ok && count) ok = fwrite(&primes[0], sizeof(uint32_t), 1, f) == 1;
    for (uint32_t i = 1; ok && i < count; i++) {
        if (primes[i] <= primes[i - 1] || primes[i] - primes[i - 1] > 0xFFFFu) { ok = false; break; }
        const uint32_t gap = primes[i] - primes[i - 1];
        if (gap > 255u) {
            const unsigned char e[3] = {0, (unsigned char)(gap & 0xFF), (unsigned char)(gap >> 8)};
            ok = fwrite(e, 1, 3, f) == 3;
        } else {
            const unsigned char g = (unsigned char)gap;
            ok = fwrite(&g, 1, 1, f) == 1;
        }
    }
    if (fclose(f) != 0) ok = false;
    return ok ? 0 : -1;
}
