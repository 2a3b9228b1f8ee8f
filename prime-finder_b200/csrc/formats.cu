// Text formats of the reference's runs (pfb_formats.h).  Host code.
#include <stdio.h>

#include "common.cuh"
#include "pfb_formats.h"

extern "C" long long pfb_read_candidates(const char *path, pfb_candidate_t *out, long long cap) {
    if (!path || cap < 0 || (cap > 0 && !out)) {
        pfb::set_error("pfb_read_candidates: bad argument");
        return PFB_E_ARG;
    }
    FILE *f = fopen(path, "r");
    if (!f) {
        pfb::set_error("pfb_read_candidates: cannot open %s", path);
        return PFB_E_IO;
    }
    long long n = 0;
    pfb_candidate_t r;
    while (fscanf(f, "%lld %lld %lld %d %d", &r.a, &r.b, &r.c, &r.k, &r.j) == 5) {
        if (n < cap) out[n] = r;
        n++;
    }
    fclose(f);
    return n;
}

static long long write_lines(const char *path, const pfb_phase2_record_t *recs, long long n, int append,
                             bool phase2) {
    if (!path || n < 0 || (n > 0 && !recs)) {
        pfb::set_error("pfb_write_phase%d: bad argument", phase2 ? 2 : 1);
        return PFB_E_ARG;
    }
    FILE *f = fopen(path, append ? "a" : "w");
    if (!f) {
        pfb::set_error("pfb_write_phase%d: cannot open %s", phase2 ? 2 : 1, path);
        return PFB_E_IO;
    }
    long long lines = 0;
    bool ok = true;
    for (long long i = 0; i < n && ok; i++) {
        const pfb_phase2_record_t &r = recs[i];
        const char *tag = nullptr;
        if (phase2) {
            if (r.result == 2) tag = " PROBABLE_PRIME_BOTH";
            else if (r.result == 3) tag = " PRIME";
            else continue;
        }
        ok = fprintf(f, "a=%lld b=%lld c=%lld k=%d j=%d%s\n", r.a, r.b, r.c, r.k, r.j, tag ? tag : "") > 0;
        lines++;
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok) {
        pfb::set_error("pfb_write_phase%d: write to %s failed", phase2 ? 2 : 1, path);
        return PFB_E_IO;
    }
    return lines;
}

extern "C" long long pfb_write_phase1(const char *path, const pfb_phase2_record_t *recs, long long n, int append) {
    return write_lines(path, recs, n, append, false);
}

extern "C" long long pfb_write_phase2(const char *path, const pfb_phase2_record_t *recs, long long n, int append) {
    return write_lines(path, recs, n, append, true);
}
