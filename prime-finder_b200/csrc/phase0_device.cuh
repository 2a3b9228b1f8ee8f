// Device side of the Phase-0 periodic table (phase0.cu): the table layout,
// the build and apply kernels, and the host construction of the table's
// entries.  Included by phase0.cu; kept apart from the host API so that the
// kernels can also be compiled for the host and run on CPU threads in the
// tests.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

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

inline uint32_t powmod_u32(uint32_t b, uint32_t e, uint32_t p) {
    uint64_t r = 1 % p, x = b % p;
    while (e) {
        if (e & 1u) r = r * x % p;
        x = x * x % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

// The tabled primes (p >= 3, 10 invertible, L = ord_p(10) <= kMaxL) with
// their first mask index and table word, and per prime the powers 10^r and
// 10^-r mod p for r < L (zero-padded to kMaxL); cells = masks, words = table
// words of all of them.
inline void phase0_tables(const uint32_t *primes, uint32_t n_primes, std::vector<Entry> &ent,
                          std::vector<uint32_t> &pw, std::vector<uint32_t> &ipw, long long &cells,
                          long long &words) {
    cells = 0;
    words = 0;
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
}

}  // namespace
