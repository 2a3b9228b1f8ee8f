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

namespace {

constexpr int kWords = 313;       // 100 x 100 bits
constexpr int kMaxL = 64;         // L^3 <= 2^18
constexpr int kBuildThreads = 128;
constexpr int kApplyThreads = 320;

struct Entry {
    uint32_t p;
    uint32_t L;
    long long cell0;     // first global mask index of this prime
    long long word0;     // first table word of this prime
};

__device__ __forceinline__ void set_bit(uint32_t *m, int bit) { atomicOr(&m[bit >> 5], 1u << (bit & 31)); }

__global__ void __launch_bounds__(kBuildThreads)
build_kernel(const Entry *__restrict__ ent, int n_ent, const uint32_t *__restrict__ pw,
             const uint32_t *__restrict__ ipw, long long total, uint32_t *__restrict__ table) {
    __shared__ uint32_t m[kWords];
    for (long long g = blockIdx.x; g < total; g += gridDim.x) {
        int e = 0;
        while (e + 1 < n_ent && ent[e + 1].cell0 <= g) e++;
        const uint32_t p = ent[e].p, L = ent[e].L;
        const long long cell = g - ent[e].cell0;
        const uint32_t rc = (uint32_t)(cell % L), rb = (uint32_t)((cell / L) % L), ra = (uint32_t)(cell / L / L);
        const uint32_t *P = pw + (size_t)e * kMaxL, *I = ipw + (size_t)e * kMaxL;
        for (int w = threadIdx.x; w < kWords; w += blockDim.x) m[w] = 0u;
        __syncthreads();
        if (threadIdx.x < 100) {
            // 64-bit arithmetic: the list may hold primes up to 2^32
            using u64 = unsigned long long;
            const u64 k = threadIdx.x + 1, pp = p;
            const int row = (int)(k - 1) * 100;
            // N form
            {
                const u64 num = ((u64)P[ra] + 2ull * pp - (k * P[rb]) % pp - 1ull) % pp;
                u64 j = num * I[rc] % pp;
                if (j == 0ull) j = pp;
                for (; j <= 100ull; j += pp) set_bit(m, row + (int)j - 1);
            }
            // rev form
            const u64 lk = k < 10ull ? 1ull : k < 100ull ? 2ull : 3ull;
            const u64 rk = lk == 1ull ? k : lk == 2ull ? (k % 10ull) * 10ull + k / 10ull : 1ull;
            const u64 rb_rev = (u64)P[ra] * I[(rb + lk) % L] % pp;
            const u64 base = ((u64)P[ra] + 2ull * pp - (rk * rb_rev) % pp - 1ull) % pp;
            const u64 c1 = (u64)I[ra] * P[(rc + 1u) % L] % pp, c2 = (u64)I[ra] * P[(rc + 2u) % L] % pp;
            const u64 r3 = (u64)P[ra] * I[(rc + 3u) % L] % pp;
            if (c1 != 0ull) {
                u64 j = base * c1 % pp;
                if (j == 0ull) j = pp;
                for (; j <= 9ull; j += pp) set_bit(m, row + (int)j - 1);
            }
            if (c2 != 0ull) {
                u64 rj = base * c2 % pp;
                if (rj == 0ull) rj = pp;
                for (; rj <= 99ull; rj += pp) {
                    int j = -1;
                    if (rj <= 9ull) j = (int)rj * 10;
                    else if (rj % 10ull != 0ull) j = (int)(rj % 10ull) * 10 + (int)(rj / 10ull);
                    if (j >= 10 && j <= 99) set_bit(m, row + j - 1);
                }
            }
            if (r3 != 0ull && r3 == base) set_bit(m, row + 99);
        }
        __syncthreads();
        uint32_t *dst = table + ent[e].word0 + cell * kWords;
        for (int w = threadIdx.x; w < kWords; w += blockDim.x) dst[w] = m[w];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kApplyThreads)
apply_kernel(const Entry *__restrict__ ent, int n_ent, const uint32_t *__restrict__ table,
             const long long *__restrict__ abc, uint32_t *__restrict__ masks, int or_in) {
    const int t = blockIdx.x, w = threadIdx.x;
    const long long a = abc[3 * t], b = abc[3 * t + 1], c = abc[3 * t + 2];
    if (w >= kWords) return;
    uint32_t acc = 0u;
    for (int e = 0; e < n_ent; e++) {
        const long long L = ent[e].L;
        const long long cell = ((a % L) * L + b % L) * L + c % L;
        acc |= __ldg(table + ent[e].word0 + cell * kWords + w);
    }
    uint32_t *out = masks + (size_t)t * kWords;
    out[w] = or_in ? (out[w] | acc) : acc;
}

uint32_t powmod_u32(uint32_t b, uint32_t e, uint32_t p) {
    uint64_t r = 1 % p, x = b % p;
    while (e) {
        if (e & 1u) r = r * x % p;
        x = x * x % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

}  // namespace

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
    // tabled primes: p >= 3, 10 invertible, L = ord_p(10) with L^3 <= 2^18
    std::vector<Entry> ent;
    std::vector<uint32_t> pw, ipw;
    long long cells = 0, words = 0;
    for (uint32_t i = 0; i < n_primes; i++) {
        const uint32_t p = primes[i];
        if (p < 3u) continue;
        uint32_t L = 0;
        uint64_t x = 10u % p;
        for (uint32_t r = 1; r <= (uint32_t)kMaxL; r++) {
            if (x == 1u) {
                L = r;
                break;
            }
            x = x * 10u % p;
        }
        if (L == 0u) continue;
        ent.push_back(Entry{p, L, cells, words});
        const uint32_t inv10 = powmod_u32(10u, p - 2u, p);  // p prime
        uint64_t a = 1, ai = 1;
        for (int r = 0; r < kMaxL; r++) {
            pw.push_back((uint32_t)(r < (int)L ? a : 0u));
            ipw.push_back((uint32_t)(r < (int)L ? ai : 0u));
            a = a * 10u % p;
            ai = ai * inv10 % p;
        }
        cells += (long long)L * L * L;
        words += (long long)L * L * L * kWords;
    }
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
