// Phase-1 trial-division sieve for sm_100a.
//
// Work of trial_div_kernel (trial_div.cu:82-159) and of the CPU twin
// sieve_one_prime (trial_div_cpu.c:32-102), re-designed for a K x K grid
// (K <= 9999) and the B200:
//
//  * Per prime and triple the eliminated (k,j) lie on straight lines:
//      N form    j   == AN - k * BN              (mod p)
//      rev form  rev(j) == AR[lj] - rev(k) * BR[lk][lj]  (mod p), one line per
//                pair of digit counts (lk, lj) of k and j.
//    AN, BN, AR, BR are products of powers of 10 and 10^-1 mod p; 10^-1 mod p
//    has a closed form, so no Fermat inversion is needed (the reference
//    inverts with powmod(x, p-2, p), trial_div.cu:107).  For p coprime to
//    10 the rev lines of all digit classes are one line, y == ar - x br, at
//    x = rev_D(k), y = rev_D(j) (D = digits of K; sieve_device.cuh).
//  * Small primes (p < S, S = max(4096, 10^digits(K))) hit many cells per row.
//    They are sieved row-tile by row-tile in shared memory; primes below 512
//    use one warp per (prime,row) so the 3333 hits of p = 3 in a row are
//    spread over 32 lanes.  The finished tile is OR-ed into global memory
//    with coalesced 32-bit atomics.
//  * Large primes (p >= S) hit each row at most once.  Their two lines are
//    enumerated by lattice walks (O(log p) per line plus O(1) per hit): a
//    warp per prime below (K^2 + X^2) / 12288 (lanes split the range of x),
//    a thread per prime above; hits are OR-ed into global memory.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "pfb_sieve.h"
#include "trial_div.h"

namespace pfb {

static thread_local char g_err[512];

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
    set_error("CUDA error %s (%s) at %s:%d: %s", cudaGetErrorName(e), cudaGetErrorString(e),
              file, line, what);
    return PFB_E_CUDA;
}

}  // namespace pfb

extern "C" const char *pfb_last_error(void) { return pfb::g_err; }

#include "sieve_device.cuh"

// ============================================================================
// Host side
// ============================================================================

struct pfb_sieve {
    int device = 0;
    uint32_t n_primes = 0;
    uint32_t s_limit = 0;  // small/large split of the last run's K
    uint32_t *d_primes = nullptr;
    uint32_t *d_tiny = nullptr, *d_small = nullptr;
    uint32_t *d_counts = nullptr;  // [tiny, small]
    uint32_t h_counts[2] = {0, 0};
    uint32_t cap_small = 0;        // capacity of d_tiny / d_small
    SmallRec *d_rec = nullptr;
    size_t rec_bytes = 0;
    long long *d_abc = nullptr;
    int abc_cap = 0;
    uint32_t *d_chunk = nullptr;
    uint32_t chunk_cap = 0;
    uint32_t *d_total = nullptr;
    uint8_t *d_stage = nullptr;    // device mask for host-mask runs
    size_t stage_bytes = 0;
    cudaStream_t stream = nullptr;
    int max_grid = 0;
};

namespace {

// The primes at or above the small limit: the medium kernel (a warp per
// prime) below medium_limit, the large kernel (a thread per prime) above;
// the digit count D of K is a template argument of both.
template <int D>
void enqueue_large_d(const uint32_t *primes, uint32_t n, uint32_t s_limit, const long long *abc, int n_abc,
                     int K, uint32_t *mask, size_t wpt, int sms, cudaStream_t st) {
    const uint32_t p_med = medium_limit(K, s_limit);
    if (p_med > s_limit)
        medium_kernel<D><<<dim3((unsigned)sms * 4u, (unsigned)n_abc), kBlockLarge, 0, st>>>(
            primes, n, s_limit, p_med, abc, K, mask, wpt);
    const unsigned blocks = (n + kBlockLarge - 1u) / kBlockLarge;
    large_kernel<D><<<dim3(blocks, (unsigned)n_abc), kBlockLarge, 0, st>>>(primes, n, p_med, abc, K, mask, wpt);
}

cudaError_t enqueue_large(const uint32_t *primes, uint32_t n, uint32_t s_limit, const long long *abc, int n_abc,
                          int K, uint32_t *mask, size_t wpt, int sms, cudaStream_t st) {
    switch (ndigits(K)) {
    case 1: enqueue_large_d<1>(primes, n, s_limit, abc, n_abc, K, mask, wpt, sms, st); break;
    case 2: enqueue_large_d<2>(primes, n, s_limit, abc, n_abc, K, mask, wpt, sms, st); break;
    case 3: enqueue_large_d<3>(primes, n, s_limit, abc, n_abc, K, mask, wpt, sms, st); break;
    default: enqueue_large_d<4>(primes, n, s_limit, abc, n_abc, K, mask, wpt, sms, st); break;
    }
    return cudaGetLastError();
}

int ensure_split(pfb_sieve *s, int K) {
    const uint32_t lim = small_limit(K);
    if (lim == s->s_limit) return PFB_OK;
    // every small prime is below lim, hence at most lim/2 of them (odd) + 1
    const uint32_t cap = lim / 2u + 2u;
    if (cap > s->cap_small) {
        cudaFree(s->d_tiny);
        cudaFree(s->d_small);
        s->d_tiny = s->d_small = nullptr;
        PFB_CUDA(cudaMalloc(&s->d_tiny, sizeof(uint32_t) * cap));
        PFB_CUDA(cudaMalloc(&s->d_small, sizeof(uint32_t) * cap));
        s->cap_small = cap;
    }
    PFB_CUDA(cudaMemsetAsync(s->d_counts, 0, 2 * sizeof(uint32_t), s->stream));
    if (s->n_primes) {
        const int blocks = (int)((s->n_primes + 255u) / 256u);
        split_kernel<<<blocks < s->max_grid ? blocks : s->max_grid, 256, 0, s->stream>>>(
            s->d_primes, s->n_primes, lim, cap, s->d_tiny, s->d_small, s->d_counts);
        PFB_CUDA(cudaGetLastError());
    }
    PFB_CUDA(cudaMemcpyAsync(s->h_counts, s->d_counts, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             s->stream));
    PFB_CUDA(cudaStreamSynchronize(s->stream));
    if (s->h_counts[0] > cap || s->h_counts[1] > cap) {
        pfb::set_error("prime list has repeated entries below %u", lim);
        return PFB_E_ARG;
    }
    s->s_limit = lim;
    return PFB_OK;
}

int set_primes(pfb_sieve *s, const uint32_t *primes, uint32_t n, bool primes_on_device,
               cudaStream_t st) {
    if (n > s->n_primes || !s->d_primes) {
        cudaFree(s->d_primes);
        s->d_primes = nullptr;
        PFB_CUDA(cudaMalloc(&s->d_primes, sizeof(uint32_t) * (n ? n : 1)));
    }
    s->n_primes = n;
    if (n)
        PFB_CUDA(cudaMemcpyAsync(s->d_primes, primes, sizeof(uint32_t) * n,
                                 primes_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    s->s_limit = 0;  // force a new split
    return PFB_OK;
}

int sieve_init(pfb_sieve *s, int device) {
    s->device = device;
    PFB_CUDA(cudaSetDevice(device));
    int sms = 0;
    PFB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    s->max_grid = sms * 16;
    PFB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    PFB_CUDA(cudaMalloc(&s->d_counts, 2 * sizeof(uint32_t)));
    PFB_CUDA(cudaMalloc(&s->d_total, sizeof(uint32_t)));
    PFB_CUDA(cudaFuncSetAttribute(small_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)tile_smem_bytes(kTileRows, PFB_SIEVE_MAX_K)));
    return PFB_OK;
}

void sieve_free(pfb_sieve *s) {
    cudaFree(s->d_primes);
    cudaFree(s->d_tiny);
    cudaFree(s->d_small);
    cudaFree(s->d_counts);
    cudaFree(s->d_rec);
    cudaFree(s->d_abc);
    cudaFree(s->d_chunk);
    cudaFree(s->d_total);
    cudaFree(s->d_stage);
    if (s->stream) cudaStreamDestroy(s->stream);
}

// Enqueue the sieve of n_abc triples (device abc already in s->d_abc) into a
// device mask that is already initialised (zeroed or holding OR-in bits).
int enqueue_sieve(pfb_sieve *s, int n_abc, int K, uint32_t *d_mask, cudaStream_t st) {
    int rc = ensure_split(s, K);
    if (rc) return rc;
    const size_t wpt = (size_t)pfb_sieve_mask_bytes(K) / 4;
    const uint32_t n_small_all = s->h_counts[0] + s->h_counts[1];
    if (n_small_all) {
        const uint32_t cap = 2u * s->cap_small;  // per-triple record stride (tiny + small lists)
        const size_t need = (size_t)n_abc * cap * sizeof(SmallRec);
        if (need > s->rec_bytes) {
            cudaFree(s->d_rec);
            s->d_rec = nullptr;
            PFB_CUDA(cudaMalloc(&s->d_rec, need));
            s->rec_bytes = need;
        }
        dim3 g1((n_small_all + 127u) / 128u, (unsigned)n_abc);
        small_setup_kernel<<<g1, 128, 0, st>>>(s->d_tiny, s->d_small, s->d_counts, s->d_abc, n_abc, K, cap,
                                               s->d_rec);
        PFB_CUDA(cudaGetLastError());
        const uint32_t tiles = ((uint32_t)K + kTileRows - 1u) / kTileRows;
        const uint32_t max_rows = (uint32_t)K < (uint32_t)kTileRows ? (uint32_t)K : (uint32_t)kTileRows;
        const size_t smem = tile_smem_bytes(max_rows, K);
        dim3 g2(tiles, (unsigned)n_abc);
        small_tile_kernel<<<g2, kBlockTile, smem, st>>>(s->d_rec, s->d_counts, cap, s->d_abc, K, d_mask, wpt);
        PFB_CUDA(cudaGetLastError());
    }
    if (s->n_primes)
        PFB_CUDA(enqueue_large(s->d_primes, s->n_primes, s->s_limit, s->d_abc, n_abc, K, d_mask, wpt,
                               s->max_grid / 16, st));
    return PFB_OK;
}

bool valid_abc(const long long *abc, int n) {
    for (int i = 0; i < 3 * n; i++)
        if (abc[i] < 0) return false;
    return true;
}

}  // namespace

extern "C" size_t pfb_sieve_mask_bytes(int K) {
    if (K <= 0) return 0;
    return (((size_t)K * (size_t)K + 31u) / 32u) * 4u;
}

extern "C" int pfb_sieve_create(pfb_sieve_t **out, const uint32_t *primes, uint32_t n_primes, int device) {
    if (!out || (n_primes && !primes)) {
        pfb::set_error("pfb_sieve_create: null argument");
        return PFB_E_ARG;
    }
    *out = nullptr;
    pfb_sieve *s = new pfb_sieve();
    int rc = sieve_init(s, device);
    if (!rc) rc = set_primes(s, primes, n_primes, false, s->stream);
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) rc = pfb::cuda_fail(e, "create sync", __FILE__, __LINE__);
    }
    if (rc) {
        sieve_free(s);
        delete s;
        return rc;
    }
    *out = s;
    return PFB_OK;
}

extern "C" void pfb_sieve_destroy(pfb_sieve_t *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    sieve_free(s);
    delete s;
}

extern "C" int pfb_sieve_run(pfb_sieve_t *s, const long long *abc, int n_abc, int K, uint8_t *mask,
                             unsigned flags, void *stream) {
    if (!s || !abc || !mask || n_abc <= 0 || n_abc > 65535 || K < 1 || K > PFB_SIEVE_MAX_K) {
        pfb::set_error("pfb_sieve_run: bad argument (n_abc=%d K=%d)", n_abc, K);
        return PFB_E_ARG;
    }
    if (!valid_abc(abc, n_abc)) {
        pfb::set_error("pfb_sieve_run: a, b, c must be >= 0");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    if (n_abc > s->abc_cap) {
        cudaFree(s->d_abc);
        s->d_abc = nullptr;
        PFB_CUDA(cudaMalloc(&s->d_abc, sizeof(long long) * 3 * n_abc));
        s->abc_cap = n_abc;
    }
    // ensure_split runs on the context stream and synchronises it, which
    // orders it before st.  A new K re-splits the prime list in place, so
    // earlier work queued on another stream (still reading the lists) must
    // finish first.
    if (small_limit(K) != s->s_limit && st != s->stream) PFB_CUDA(cudaStreamSynchronize(st));
    int rc = ensure_split(s, K);
    if (rc) return rc;
    PFB_CUDA(cudaMemcpyAsync(s->d_abc, abc, sizeof(long long) * 3 * n_abc, cudaMemcpyHostToDevice, st));
    const size_t blk = pfb_sieve_mask_bytes(K);
    const size_t total = blk * (size_t)n_abc;
    uint32_t *d_mask = (uint32_t *)mask;
    const bool host = (flags & PFB_SIEVE_MASK_HOST) != 0;
    if (host) {
        if (total > s->stage_bytes) {
            cudaFree(s->d_stage);
            s->d_stage = nullptr;
            PFB_CUDA(cudaMalloc(&s->d_stage, total));
            s->stage_bytes = total;
        }
        d_mask = (uint32_t *)s->d_stage;
        if (flags & PFB_SIEVE_OR)
            PFB_CUDA(cudaMemcpyAsync(d_mask, mask, total, cudaMemcpyHostToDevice, st));
        else
            PFB_CUDA(cudaMemsetAsync(d_mask, 0, total, st));
    } else if (!(flags & PFB_SIEVE_OR)) {
        PFB_CUDA(cudaMemsetAsync(d_mask, 0, total, st));
    }
    rc = enqueue_sieve(s, n_abc, K, d_mask, st);
    if (rc) return rc;
    if (host) {
        PFB_CUDA(cudaMemcpyAsync(mask, d_mask, total, cudaMemcpyDeviceToHost, st));
        PFB_CUDA(cudaStreamSynchronize(st));
    }
    return PFB_OK;
}

extern "C" int pfb_sieve_survivors(pfb_sieve_t *s, const uint8_t *d_mask, int K, uint32_t *d_out,
                                   uint32_t cap, uint32_t *count, void *stream) {
    if (!s || !d_mask || !count || K < 1 || K > PFB_SIEVE_MAX_K) {
        pfb::set_error("pfb_sieve_survivors: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    const uint32_t nbits = (uint32_t)K * (uint32_t)K;
    const uint32_t nwords = (nbits + 31u) / 32u;
    const uint32_t chunks = (nwords + 31u) / 32u;
    if (chunks > s->chunk_cap) {
        cudaFree(s->d_chunk);
        s->d_chunk = nullptr;
        PFB_CUDA(cudaMalloc(&s->d_chunk, sizeof(uint32_t) * chunks));
        s->chunk_cap = chunks;
    }
    surv_count_kernel<<<chunks, 32, 0, st>>>((const uint32_t *)d_mask, nbits, s->d_chunk);
    PFB_CUDA(cudaGetLastError());
    surv_scan_kernel<<<1, 1024, 0, st>>>(s->d_chunk, chunks, s->d_total);
    PFB_CUDA(cudaGetLastError());
    surv_write_kernel<<<chunks, 32, 0, st>>>((const uint32_t *)d_mask, nbits, K, s->d_chunk, d_out, cap);
    PFB_CUDA(cudaGetLastError());
    PFB_CUDA(cudaMemcpyAsync(count, s->d_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    PFB_CUDA(cudaStreamSynchronize(st));
    if (*count > cap) {
        pfb::set_error("pfb_sieve_survivors: %u survivors, capacity %u", *count, cap);
        return PFB_E_CAPACITY;
    }
    return PFB_OK;
}

// ---------------------------------------------------------------------------
// Drop-in entry points of trial_div.h.  One internal context per device,
// reused across calls (the reference allocates and frees per call,
// trial_div.cu:211-257); like the reference, not thread-safe.

namespace {
std::mutex g_ctx_mu;
std::vector<pfb_sieve *> g_ctx;

int context_for_current_device(pfb_sieve **out) {
    int dev = 0;
    PFB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if ((int)g_ctx.size() <= dev) g_ctx.resize(dev + 1, nullptr);
    if (!g_ctx[dev]) {
        pfb_sieve *s = new pfb_sieve();
        int rc = sieve_init(s, dev);
        if (rc) {
            sieve_free(s);
            delete s;
            return rc;
        }
        g_ctx[dev] = s;
    }
    *out = g_ctx[dev];
    return PFB_OK;
}
}  // namespace

extern "C" int trial_div_gpu_grid(const uint32_t *primes, uint32_t n_primes, const long long *abc, int n_abc,
                                  int K, uint8_t *mask_out, unsigned flags) {
    if ((n_primes && !primes) || !abc || !mask_out || n_abc <= 0) {
        pfb::set_error("trial_div_gpu_grid: bad argument");
        return PFB_E_ARG;
    }
    pfb_sieve *s = nullptr;
    int rc = context_for_current_device(&s);
    if (rc) return rc;
    rc = set_primes(s, primes, n_primes, false, s->stream);
    if (rc) return rc;
    return pfb_sieve_run(s, abc, n_abc, K, mask_out, (flags & PFB_SIEVE_OR) | PFB_SIEVE_MASK_HOST, nullptr);
}

extern "C" int cuda_get_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

extern "C" int cuda_set_device(int index) { return cudaSetDevice(index) == cudaSuccess ? 0 : -1; }

static double event_secs(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return (double)ms * 1e-3;
}

extern "C" int trial_div_gpu(const prime_list_t *pl, long long a, long long b, long long c, uint32_t *sieve_bits,
                             gpu_timing_t *timing) {
    if (timing) *timing = gpu_timing_t{0.0, 0.0, 0.0};
    int rc = PFB_E_ARG;
    pfb_sieve *s = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    if (!pl || !sieve_bits || (pl->count && !pl->primes) || a < 0 || b < 0 || c < 0) {
        pfb::set_error("trial_div_gpu: bad argument");
        goto done;
    }
    rc = context_for_current_device(&s);
    if (rc) goto done;
    {
        cudaStream_t st = s->stream;
        for (auto &e : ev)
            if (cudaEventCreate(&e) != cudaSuccess) { rc = PFB_E_CUDA; goto done; }
        const long long abc[3] = {a, b, c};
        const size_t blk = pfb_sieve_mask_bytes(100);
        if (blk > s->stage_bytes) {
            cudaFree(s->d_stage);
            s->d_stage = nullptr;
            if (cudaMalloc(&s->d_stage, blk) != cudaSuccess) { rc = PFB_E_CUDA; goto done; }
            s->stage_bytes = blk;
        }
        if (s->abc_cap < 1) {
            if (cudaMalloc(&s->d_abc, sizeof(long long) * 3) != cudaSuccess) { rc = PFB_E_CUDA; goto done; }
            s->abc_cap = 1;
        }
        cudaEventRecord(ev[0], st);
        rc = set_primes(s, pl->primes, pl->count, false, st);
        if (rc) goto done;
        if (cudaMemcpyAsync(s->d_stage, sieve_bits, blk, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(s->d_abc, abc, sizeof(abc), cudaMemcpyHostToDevice, st) != cudaSuccess) {
            rc = PFB_E_CUDA;
            goto done;
        }
        cudaEventRecord(ev[1], st);
        rc = enqueue_sieve(s, 1, 100, (uint32_t *)s->d_stage, st);
        if (rc) goto done;
        cudaEventRecord(ev[2], st);
        if (cudaMemcpyAsync(sieve_bits, s->d_stage, blk, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
            rc = PFB_E_CUDA;
            goto done;
        }
        cudaEventRecord(ev[3], st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            rc = pfb::cuda_fail(e, "trial_div_gpu sync", __FILE__, __LINE__);
            goto done;
        }
        if (timing) {
            timing->upload = event_secs(ev[0], ev[1]);
            timing->kernel = event_secs(ev[1], ev[2]);
            timing->download = event_secs(ev[2], ev[3]);
        }
        rc = 0;
    }
done:
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    if (rc != 0) {
        fprintf(stderr, "trial_div_gpu: CUDA error (%s)\n", pfb_last_error());
        rc = -1;
    }
    return rc;
}

void trial_div_launch(const uint32_t *d_primes, uint32_t n_primes, uint64_t a, uint64_t b, uint64_t c,
                      uint32_t *d_bits, int block_size) {
    (void)block_size;
    pfb_sieve *s = nullptr;
    if (context_for_current_device(&s)) return;
    cudaStream_t st = 0;  // legacy default stream, as trial_div.cu:168
    if (set_primes(s, d_primes, n_primes, true, st)) return;
    if (cudaStreamSynchronize(st) != cudaSuccess) return;
    const long long abc[3] = {(long long)a, (long long)b, (long long)c};
    if (s->abc_cap < 1) {
        if (cudaMalloc(&s->d_abc, sizeof(long long) * 3) != cudaSuccess) return;
        s->abc_cap = 1;
    }
    if (ensure_split(s, 100)) return;
    cudaMemcpyAsync(s->d_abc, abc, sizeof(abc), cudaMemcpyHostToDevice, st);
    enqueue_sieve(s, 1, 100, d_bits, st);
}

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot call cudaMalloc: a process whose device memory is
// reserved up front by another allocator (a framework's caching allocator or
// a fixed memory pool that owns nearly all of HBM), or a latency-sensitive
// loop that cannot take the device-wide synchronisation cudaFree implies.
// pfb_sieve_run_noalloc serves them: the caller passes the prime list and the
// mask in device memory it already owns, and the working memory of the sieve
// (small-prime lists and their counts, the per-prime line records, the
// triple) lives in one file-scope __device__ array of fixed size that every
// GPU loading this library holds until the process exits.

namespace {

constexpr uint32_t kNoAllocLimit = 10000u;                   // small_limit(K) for every K <= 9999
constexpr uint32_t kNoAllocListCap = kNoAllocLimit / 2u + 2u;  // odd values below the limit, + 2
constexpr uint32_t kNoAllocSeenWords = kNoAllocLimit / 32u + 1u;

struct NoAllocScratch {
    uint32_t counts[2];
    uint32_t pad0[62];
    long long abc[4];
    uint32_t seen[kNoAllocSeenWords];  // small values already listed (bit v)
    uint32_t tiny[kNoAllocListCap];
    uint32_t small[kNoAllocListCap];
    SmallRec rec[2 * kNoAllocListCap];
};

// 361 688 bytes (0.36 MB): the scratch of one triple at any K <= 9999.
static_assert(sizeof(NoAllocScratch) == 361688, "the size the header states");
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// One block: clears the counts and the seen-bitmap, stores the triple.
__global__ void noalloc_begin_kernel(NoAllocScratch *sc, long long a, long long b, long long c) {
    for (uint32_t w = threadIdx.x; w < kNoAllocSeenWords; w += blockDim.x) sc->seen[w] = 0u;
    if (threadIdx.x == 0) {
        sc->counts[0] = 0u;
        sc->counts[1] = 0u;
        sc->abc[0] = a;
        sc->abc[1] = b;
        sc->abc[2] = c;
    }
}

std::mutex g_noalloc_mu;
NoAllocScratch *g_noalloc_ptr[128];
int g_noalloc_sms[128];

// Once per device, with that device current: the device address of the
// scratch array (in host code its name is only a host-side stand-in).
int noalloc_scratch(int dev, NoAllocScratch **out, int *sms) {
    if (dev < 0 || dev >= 128) {
        pfb::set_error("pfb_sieve_run_noalloc: device %d out of range", dev);
        return PFB_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        PFB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        int n = 0;
        PFB_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
        PFB_CUDA(cudaFuncSetAttribute(small_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)tile_smem_bytes(kTileRows, PFB_SIEVE_MAX_K)));
        g_noalloc_sms[dev] = n;
        g_noalloc_ptr[dev] = (NoAllocScratch *)p;
    }
    *out = g_noalloc_ptr[dev];
    *sms = g_noalloc_sms[dev];
    return PFB_OK;
}

}  // namespace

extern "C" int pfb_sieve_run_noalloc(const uint32_t *d_primes, uint32_t n_primes, long long a, long long b,
                                     long long c, int K, uint32_t *d_mask, unsigned flags, void *stream) {
    if ((n_primes && !d_primes) || !d_mask || a < 0 || b < 0 || c < 0) {
        pfb::set_error("pfb_sieve_run_noalloc: bad argument");
        return PFB_E_ARG;
    }
    if (K < 1 || K > PFB_SIEVE_MAX_K) {
        pfb::set_error("pfb_sieve_run_noalloc: K = %d is outside [1, %d], the size the fixed scratch holds", K,
                       PFB_SIEVE_MAX_K);
        return PFB_E_CAPACITY;
    }
    int dev = 0;
    PFB_CUDA(cudaGetDevice(&dev));
    NoAllocScratch *sc = nullptr;
    int sms = 0;
    int rc = noalloc_scratch(dev, &sc, &sms);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t wpt = pfb_sieve_mask_bytes(K) / 4;
    if (!(flags & PFB_SIEVE_OR)) PFB_CUDA(cudaMemsetAsync(d_mask, 0, wpt * 4, st));
    noalloc_begin_kernel<<<1, 320, 0, st>>>(sc, a, b, c);
    PFB_CUDA(cudaGetLastError());
    const uint32_t lim = small_limit(K);
    const uint32_t cap = kNoAllocListCap;
    if (n_primes) {
        const int blocks = (int)std::min<uint32_t>((n_primes + 255u) / 256u, (uint32_t)sms * 16u);
        split_unique_kernel<<<blocks, 256, 0, st>>>(d_primes, n_primes, lim, sc->seen, sc->tiny, sc->small,
                                                    sc->counts);
        PFB_CUDA(cudaGetLastError());
        // record stride 2*cap: tiny then small; the kernels read the counts on the device
        dim3 g1((2u * cap + 127u) / 128u, 1u);
        small_setup_kernel<<<g1, 128, 0, st>>>(sc->tiny, sc->small, sc->counts, sc->abc, 1, K, 2u * cap, sc->rec);
        PFB_CUDA(cudaGetLastError());
        const uint32_t tiles = ((uint32_t)K + kTileRows - 1u) / kTileRows;
        const uint32_t rows = (uint32_t)K < (uint32_t)kTileRows ? (uint32_t)K : (uint32_t)kTileRows;
        small_tile_kernel<<<dim3(tiles, 1u), kBlockTile, tile_smem_bytes(rows, K), st>>>(
            sc->rec, sc->counts, 2u * cap, sc->abc, K, d_mask, wpt);
        PFB_CUDA(cudaGetLastError());
        PFB_CUDA(enqueue_large(d_primes, n_primes, lim, sc->abc, 1, K, d_mask, wpt, sms, st));
    }
    return PFB_OK;
}
