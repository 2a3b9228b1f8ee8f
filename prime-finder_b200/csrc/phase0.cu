// Phase-0 periodic sieve table on the GPU (pfb_phase0.h).
//
// The masks are those of the reference's fill_prime_bitmask
// (sieve_table.c:93-178): for a tabled prime p (L = ord_p(10) <= 64) and a
// residue triple (ra, rb, rc), with P[r] = 10^r mod p and I[r] = 10^-r mod p,
//   N form:   j == (P[ra] - k P[rb] - 1) I[rc]            (mod p), j in 1..100
//   rev form: with B_k = P[ra] - rev(k) P[ra] I[(rb + lk) mod L] - 1,
//             rev(j) == B_k I[ra] P[(rc + lj) mod L]      (mod p)
//             for one-digit j (j itself), two-digit j (rev(j) in 1..99, no
//             trailing zero of rev(j)) and j = 100 (rev(j) = 1).
// One CTA builds one mask in shared memory (a thread per k) and writes it
// out coalesced; a grid-stride loop covers every mask of every prime.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "common.cuh"
#include "pfb_phase0.h"

#include "phase0_device.cuh"

struct pfb_phase0 {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n_ent = 0;
    long long n_masks = 0;
    Entry *d_ent = nullptr;
    uint32_t *d_table = nullptr;
    size_t table_bytes = 0;
    double build_s = 0.0;
};

static void phase0_free(pfb_phase0 *t) {
    if (!t) return;
    if (t->d_ent) cudaFree(t->d_ent);
    if (t->d_table) cudaFree(t->d_table);
    if (t->stream) cudaStreamDestroy(t->stream);
    delete t;
}

extern "C" int pfb_phase0_create(pfb_phase0_t **out, const uint32_t *primes, uint32_t n_primes, int device) {
    if (!out || (n_primes && !primes)) {
        pfb::set_error("pfb_phase0_create: bad argument");
        return PFB_E_ARG;
    }
    *out = nullptr;
    std::vector<Entry> ent;
    std::vector<uint32_t> pw, ipw;
    long long cells = 0, words = 0;
    phase0_tables(primes, n_primes, ent, pw, ipw, cells, words);
    pfb_phase0 *t = new pfb_phase0();
    t->device = device;
    t->n_ent = (int)ent.size();
    t->n_masks = cells;
    t->table_bytes = (size_t)words * sizeof(uint32_t);
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t ce = cudaSetDevice(device);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
        phase0_free(t);
        return pfb::cuda_fail(ce, "phase0 stream", __FILE__, __LINE__);
    }
    if (t->n_ent > 0) {
        uint32_t *d_pw = nullptr;
        if (cudaMalloc(&t->d_table, t->table_bytes) != cudaSuccess ||
            cudaMalloc(&t->d_ent, ent.size() * sizeof(Entry)) != cudaSuccess ||
            cudaMalloc(&d_pw, 2 * pw.size() * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            if (d_pw) cudaFree(d_pw);
            pfb::set_error("pfb_phase0_create: cannot allocate %zu bytes of device memory", t->table_bytes);
            phase0_free(t);
            return PFB_E_NOMEM;
        }
        ce = cudaMemcpyAsync(t->d_ent, ent.data(), ent.size() * sizeof(Entry), cudaMemcpyHostToDevice, t->stream);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(d_pw, pw.data(), pw.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, t->stream);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(d_pw + pw.size(), ipw.data(), ipw.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                 t->stream);
        if (ce == cudaSuccess) {
            int sms = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            const long long grid = std::min<long long>(cells, (long long)std::max(1, sms) * 16);
            build_kernel<<<(unsigned)grid, kBuildThreads, 0, t->stream>>>(t->d_ent, t->n_ent, d_pw, d_pw + pw.size(),
                                                                          cells, t->d_table);
            ce = cudaGetLastError();
        }
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(t->stream);
        cudaFree(d_pw);
        if (ce != cudaSuccess) {
            phase0_free(t);
            return pfb::cuda_fail(ce, "phase0 build", __FILE__, __LINE__);
        }
    }
    t->build_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = t;
    return PFB_OK;
}

extern "C" int pfb_phase0_apply(pfb_phase0_t *t, const long long *abc, int n_abc, uint32_t *masks, unsigned flags,
                                void *stream) {
    if (!t || !abc || n_abc <= 0 || !masks) {
        pfb::set_error("pfb_phase0_apply: bad argument");
        return PFB_E_ARG;
    }
    for (int i = 0; i < 3 * n_abc; i++)
        if (abc[i] < 0) {
            pfb::set_error("pfb_phase0_apply: negative exponent in triple %d", i / 3);
            return PFB_E_ARG;
        }
    PFB_CUDA(cudaSetDevice(t->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : t->stream;
    const bool host = (flags & PFB_SIEVE_MASK_HOST) != 0, or_in = (flags & PFB_SIEVE_OR) != 0;
    const size_t mbytes = (size_t)n_abc * kWords * sizeof(uint32_t);
    long long *d_abc = nullptr;
    uint32_t *d_masks = masks;
    int rc = PFB_OK;
    if (cudaMalloc(&d_abc, 3 * (size_t)n_abc * sizeof(long long)) != cudaSuccess ||
        (host && cudaMalloc(&d_masks, mbytes) != cudaSuccess)) {
        cudaGetLastError();
        if (d_abc) cudaFree(d_abc);
        pfb::set_error("pfb_phase0_apply: cannot allocate device memory");
        return PFB_E_NOMEM;
    }
    cudaError_t ce = cudaMemcpyAsync(d_abc, abc, 3 * (size_t)n_abc * sizeof(long long), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && host && or_in) ce = cudaMemcpyAsync(d_masks, masks, mbytes, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) {
        if (t->n_ent > 0) {
            apply_kernel<<<n_abc, kApplyThreads, 0, st>>>(t->d_ent, t->n_ent, t->d_table, d_abc, d_masks, or_in);
            ce = cudaGetLastError();
        } else if (!or_in) {
            ce = cudaMemsetAsync(d_masks, 0, mbytes, st);
        }
    }
    if (ce == cudaSuccess && host) ce = cudaMemcpyAsync(masks, d_masks, mbytes, cudaMemcpyDeviceToHost, st);
    // the argument copy must finish before it is freed
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "phase0 apply", __FILE__, __LINE__);
    cudaFree(d_abc);
    if (host) cudaFree(d_masks);
    return rc;
}

extern "C" int pfb_phase0_info(pfb_phase0_t *t, int *n_primes, long long *n_masks, size_t *table_bytes,
                               double *build_seconds) {
    if (!t) {
        pfb::set_error("pfb_phase0_info: null table");
        return PFB_E_ARG;
    }
    if (n_primes) *n_primes = t->n_ent;
    if (n_masks) *n_masks = t->n_masks;
    if (table_bytes) *table_bytes = t->table_bytes;
    if (build_seconds) *build_seconds = t->build_s;
    return PFB_OK;
}

extern "C" void pfb_phase0_destroy(pfb_phase0_t *t) {
    if (!t) return;
    cudaSetDevice(t->device);
    if (t->stream) cudaStreamSynchronize(t->stream);
    phase0_free(t);
}
