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
//    inverts with powmod(x, p-2, p), trial_div.cu:107).
//  * Small primes (p < S, S = max(4096, 10^digits(K))) hit many cells per row.
//    They are sieved row-tile by row-tile in shared memory; primes below 512
//    use one warp per (prime,row) so the 3333 hits of p = 3 in a row are
//    spread over 32 lanes.  The finished tile is OR-ed into global memory
//    with coalesced 32-bit atomics.
//  * Large primes (p >= S) hit each row at most once.  One thread per prime
//    enumerates the hits of its long lines with a lattice walk (O(log p) per
//    line plus O(1) per hit), iterates the short lines (<= 99 values on one
//    side) with incremental modular updates, and OR-s the hits into global
//    memory.
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

namespace {

using pfb::Mod32;

constexpr uint32_t kTinyLimit = 512;      // primes below: one warp per (prime,row)
constexpr int kTileRows = 64;             // rows of the (k,j) grid per shared-memory tile
constexpr int kBlockTile = 512;
constexpr int kBlockLarge = 256;

__host__ __device__ inline int ndigits(int x) { return x < 10 ? 1 : x < 100 ? 2 : x < 1000 ? 3 : 4; }
__host__ __device__ inline uint32_t pow10i(int d) {
    return d == 0 ? 1u : d == 1 ? 10u : d == 2 ? 100u : d == 3 ? 1000u : 10000u;
}
// Decimal reversal of x written with exactly l digits (miller_rabin.c:45-54).
__device__ __forceinline__ uint32_t rev_digits(uint32_t x, int l) {
    uint32_t r = 0;
    for (int i = 0; i < l; i++) {
        uint32_t q = x / 10u;
        r = r * 10u + (x - q * 10u);
        x = q;
    }
    return r;
}

// Shared-memory words of a tile of `rows` grid rows: the bit range may start
// and end inside a word, hence the two extra words.
inline size_t tile_smem_bytes(uint32_t rows, int K) {
    return (((size_t)rows * (size_t)K + 31u) / 32u + 2u) * sizeof(uint32_t);
}

inline uint32_t small_limit(int K) {
    uint32_t s = pow10i(ndigits(K));
    return s > 4096u ? s : 4096u;
}

// Per (prime, triple) line coefficients.  flags: bit 0 = N form active,
// bit lk = rev k-class lk active (1..4), bit 4+lj = rev j-class lj active.
struct LineConsts {
    uint32_t an, bn;
    uint32_t ar[4];
    uint32_t br[4][4];
    uint32_t flags;
};

// Small-prime record kept in global memory between the set-up kernel and
// the tile kernel.
struct SmallRec {
    uint32_t p;
    uint32_t m_lo, m_hi;
    LineConsts lc;
};

__device__ void line_consts(const Mod32 &M, long long a, long long b, long long c, LineConsts &s) {
    const uint32_t p = M.p;
    const bool inv_ok = (p & 1u) && (p % 5u != 0u);
    const uint32_t ten = 10u % p;
    uint32_t inv10 = 0;
    if (inv_ok) {
        uint32_t d = p % 10u;
        uint32_t t = d == 1 ? 9u : d == 3 ? 3u : d == 7 ? 7u : 1u;
        inv10 = (uint32_t)(((unsigned long long)p * t + 1ull) / 10ull);
    }
    // 10^e mod p (e >= 0) and 10^-e mod p (only when 10 is invertible).  When
    // p is 2 or 5, 10^e is 1 for e == 0 and 0 otherwise, and 1 is its own
    // inverse: every coefficient below then reduces to 0 or 1 consistently.
    auto pw = [&](long long e) -> uint32_t { return inv_ok ? M.pow(ten, (unsigned long long)e) : (e == 0 ? 1u : 0u); };
    auto ipw = [&](long long e) -> uint32_t { return inv_ok ? M.pow(inv10, (unsigned long long)e) : (e == 0 ? 1u : 0u); };

    s.flags = 0;
    const uint32_t ra = pw(a);
    const uint32_t ram1 = M.sub(ra, 1u);
    // N form: j * 10^c == 10^a - 1 - k * 10^b  (trial_div_cpu.c:40-52).
    if (inv_ok || c == 0) {
        const uint32_t inv_rc = ipw(c);
        s.an = M.mul(ram1, inv_rc);
        s.bn = inv_ok ? (b >= c ? pw(b - c) : ipw(c - b)) : M.mul(pw(b), inv_rc);
        s.flags |= 1u;
    } else {
        s.an = s.bn = 0;
    }
    // rev form (trial_div_cpu.c:54-101): rb_rev[l] = 10^(a-b-l), rc_rev[l] = 10^(a-c-l),
    // a class is skipped when its exponent is negative or its power is 0 mod p.
    uint32_t rbr[4], irc[4];
    {
        const long long e4 = a - b - 4;
        uint32_t base = e4 >= 0 ? pw(e4) : 0u;
        for (int l = 4; l >= 1; l--) {
            const long long e = a - b - l;
            const bool ok = e >= 0 && (inv_ok || e == 0);
            if (ok) {
                rbr[l - 1] = (e4 >= 0) ? base : pw(e);
                s.flags |= 1u << l;
            } else {
                rbr[l - 1] = 0;
            }
            if (e4 >= 0) base = M.mul(base, ten);
        }
    }
    {
        const long long f1 = a - c - 1;
        uint32_t q = (inv_ok && f1 >= 0) ? ipw(f1) : 0u;
        for (int l = 1; l <= 4; l++) {
            const long long e = a - c - l;
            const bool ok = e >= 0 && (inv_ok || e == 0);
            if (ok) {
                irc[l - 1] = inv_ok ? q : 1u;
                s.flags |= 1u << (4 + l);
            } else {
                irc[l - 1] = 0;
            }
            if (inv_ok) q = M.mul(q, ten);
        }
    }
    for (int lj = 0; lj < 4; lj++) {
        s.ar[lj] = M.mul(ram1, irc[lj]);
        for (int lk = 0; lk < 4; lk++) s.br[lk][lj] = M.mul(rbr[lk], irc[lj]);
    }
}

__device__ __forceinline__ void mark_global(uint32_t *mask, int K, uint32_t k, uint32_t j) {
    const uint32_t q = (k - 1u) * (uint32_t)K + (j - 1u);
    atomicOr(mask + (q >> 5), 1u << (q & 31u));
}

// ---------------------------------------------------------------------------
// Lattice enumeration of one line.  The hits of y == A - B x (mod p) with x in
// [x0, x1] and 1 <= y <= Y (Y < p) are the points of a translate of the
// lattice {(i, t) : i == g t (mod p)}, g = -B, that fall in the strip
// 0 <= i < Y (i = y - 1, t = x - x0).
//
//  * first_hit: the smallest t >= 0 with (c + g t) mod p < Y, by a Euclid-like
//    descent on (multiplier, modulus) that halves the modulus every level
//    (reflection keeps the multiplier below half the modulus): depth <= 33.
//  * fk_reduce: a basis u = (-a, beta), v = (c, delta) with 0 <= a, c < Y,
//    a + c >= Y, beta, delta > 0 (Franke and Kleinjung, "Continued fractions
//    and lattice sieving", 2005).  From a strip point (i, t) the next strip
//    point is (i, t) + u if i >= a, + v if i + c < Y, else + u + v.
// Cost: O(log p) per line plus O(1) per hit, where walking the K values of x
// costs O(K).

// Exact quotients by d from a double estimate (rd = 1/d, one division per
// divisor) corrected with integer arithmetic: for quotients below 2^50 the
// estimate is within two units.
__device__ __forceinline__ uint32_t quot32(uint32_t v, uint32_t d, double rd) {
    uint32_t q = (uint32_t)((double)v * rd);
    long long r = (long long)v - (long long)q * d;
    while (r < 0) {
        q--;
        r += d;
    }
    while (r >= (long long)d) {
        q++;
        r -= d;
    }
    return q;
}

__device__ __forceinline__ unsigned long long quot64(unsigned long long n, uint32_t d, double rd) {
    unsigned long long q = (unsigned long long)((double)n * rd);
    long long r = (long long)(n - q * d);
    while (r < 0) {
        q--;
        r += d;
    }
    while (r >= (long long)d) {
        q++;
        r -= d;
    }
    return q;
}

// The descent keeps, per level, the multiplier a, its reciprocal and the
// interval start L; the level's modulus is the previous level's multiplier
// (p at level 0).
__device__ __noinline__ uint32_t first_hit(uint32_t c, uint32_t g, uint32_t p, uint32_t Y) {
    if (c < Y) return 0u;
    uint32_t a = g, m = p, L = p - c, R = p - c + Y - 1u;
    uint32_t sa[34], sl[34];
    double sr[34];
    int d = 0;
    uint32_t x;
    for (;;) {
        const double rd = 1.0 / (double)a;
        const uint32_t k = quot32(L - 1u, a, rd) + 1u;  // ceil(L / a), L >= 1
        if ((unsigned long long)a * k <= R) {
            x = k;
            break;
        }
        if (d >= 34) return 0xFFFFFFFFu;  // unreachable: the modulus halves each level
        sa[d] = a;
        sl[d] = L;
        sr[d] = rd;
        d++;
        const uint32_t r = m - quot32(m, a, rd) * a;  // != 0: gcd(a, m) = 1 along the chain
        uint32_t a2 = a - r, L2 = L - quot32(L, a, rd) * a, R2 = R - quot32(R, a, rd) * a;
        const uint32_t m2 = a;
        if (a2 > (m2 >> 1)) {               // reflect: a x in [L, R] <=> (m - a) x in [m - R, m - L]
            a2 = r;
            const uint32_t t2 = m2 - R2;
            R2 = m2 - L2;
            L2 = t2;
        }
        a = a2;
        m = m2;
        L = L2;
        R = R2;
    }
    while (d > 0) {
        d--;
        const uint32_t md = d ? sa[d - 1] : p;
        x = (uint32_t)quot64((unsigned long long)x * md + sl[d] + sa[d] - 1u, sa[d], sr[d]);  // ceil
    }
    return x;
}

struct FKBasis {
    uint32_t a, beta, c, delta;
};

__device__ __noinline__ FKBasis fk_reduce(uint32_t g, uint32_t p, uint32_t I) {
    uint32_t a = p, beta = 0u, c = g, delta = 1u;
    for (;;) {
        if (c < I) {
            const uint32_t k = (a - (I - c)) / c;
            a -= k * c;
            beta += k * delta;
            break;
        }
        if (a < I) {
            const uint32_t k = (c - (I - a)) / a;
            c -= k * a;
            delta += k * beta;
            break;
        }
        if (a >= c) {
            const uint32_t k = a / c;
            a -= k * c;
            beta += k * delta;
        } else {
            const uint32_t k = c / a;
            c -= k * a;
            delta += k * beta;
        }
    }
    return FKBasis{a, beta, c, delta};
}

// Calls visit(x, y) for every x in [x0, x1] with y = (A - B x) mod p in
// [1, Y]; requires 1 <= Y < p, B != 0 (mod p), x1 - x0 < p.
template <class Visit>
__device__ __forceinline__ void line_hits(const Mod32 &M, uint32_t A, uint32_t B, uint32_t x0, uint32_t x1,
                                          uint32_t Y, Visit visit) {
    const uint32_t p = M.p;
    const uint32_t g = p - B;
    const uint32_t c0 = M.sub(M.sub(A, 1u % p), M.mul(B, x0 % p));  // (A - 1 - B x0) mod p
    unsigned long long t = first_hit(c0, g, p, Y);
    const unsigned long long span = (unsigned long long)(x1 - x0);
    if (t > span) return;
    const FKBasis fb = fk_reduce(g, p, Y);
    uint32_t i = M.red((unsigned long long)g * t + c0);
    while (t <= span) {
        visit(x0 + (uint32_t)t, i + 1u);
        if (i >= fb.a) {
            i -= fb.a;
            t += fb.beta;
        } else if (i + fb.c < Y) {
            i += fb.c;
            t += fb.delta;
        } else {
            i = i - fb.a + fb.c;
            t += (unsigned long long)fb.beta + fb.delta;
        }
    }
}

// ---------------------------------------------------------------------------
// Prime-list split: tiny (p < 512), small (512 <= p < S); large primes are
// filtered inside the large-prime kernel.
// A list with repeated entries can exceed `cap`; the excess is counted but
// not stored, and the host rejects the list.
__global__ void split_kernel(const uint32_t *__restrict__ primes, uint32_t n, uint32_t s_limit,
                             uint32_t cap, uint32_t *tiny, uint32_t *small, uint32_t *counts) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = primes[i];
        if (p < 2u || p >= s_limit) continue;
        if (p < kTinyLimit) {
            const uint32_t at = atomicAdd(&counts[0], 1u);
            if (at < cap) tiny[at] = p;
        } else {
            const uint32_t at = atomicAdd(&counts[1], 1u);
            if (at < cap) small[at] = p;
        }
    }
}

// Set-up of the small-prime records for every triple: rec[t * cap + i];
// cap = 2 * capacity of each list.
__global__ void small_setup_kernel(const uint32_t *__restrict__ tiny, const uint32_t *__restrict__ small,
                                   const uint32_t *__restrict__ counts, const long long *__restrict__ abc,
                                   int n_abc, uint32_t cap, SmallRec *__restrict__ rec) {
    const uint32_t n_tiny = min(counts[0], cap / 2u), n_small = min(counts[1], cap / 2u);
    const uint32_t n = n_tiny + n_small;
    const int t = blockIdx.y;
    if (t >= n_abc) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = i < n_tiny ? tiny[i] : small[i - n_tiny];
        Mod32 M;
        M.init(p);
        SmallRec r;
        r.p = p;
        r.m_lo = (uint32_t)M.m;
        r.m_hi = (uint32_t)(M.m >> 32);
        line_consts(M, abc[3 * t], abc[3 * t + 1], abc[3 * t + 2], r.lc);
        rec[(size_t)t * cap + i] = r;
    }
}

// Marks of one (prime,row) item.  Lanes lane0, lane0+step, ... of the hit
// sequences are handled by this thread (step = 32 for warp items, 1 for
// thread items).
__device__ __forceinline__ void small_item(const SmallRec &r, uint32_t k, int K, uint32_t lane0,
                                           uint32_t step, uint32_t *tile, uint32_t bit_base) {
    Mod32 M;
    M.p = r.p;
    M.m = ((unsigned long long)r.m_hi << 32) | r.m_lo;
    const uint32_t p = r.p;
    const LineConsts &lc = r.lc;
    auto mark = [&](uint32_t j) {
        const uint32_t q = (k - 1u) * (uint32_t)K + (j - 1u) - bit_base;
        atomicOr(tile + (q >> 5), 1u << (q & 31u));
    };
    if (lc.flags & 1u) {
        uint32_t j0 = M.sub(lc.an, M.mul(k % p, lc.bn));
        if (j0 == 0) j0 = p;
        for (unsigned long long j = j0 + (unsigned long long)lane0 * p; j <= (unsigned long long)K;
             j += (unsigned long long)step * p)
            mark((uint32_t)j);
    }
    const int lk = ndigits((int)k);
    if (!(lc.flags & (1u << lk))) return;
    const uint32_t rk = rev_digits(k, lk) % p;
    const int maxd = ndigits(K);
    for (int lj = 1; lj <= maxd; lj++) {
        if (!(lc.flags & (1u << (4 + lj)))) continue;
        const uint32_t lim = pow10i(lj);  // rj < lim
        uint32_t t0 = M.sub(lc.ar[lj - 1], M.mul(rk, lc.br[lk - 1][lj - 1]));
        if (t0 == 0) t0 = p;
        for (unsigned long long rj = t0 + (unsigned long long)lane0 * p; rj < lim;
             rj += (unsigned long long)step * p) {
            const uint32_t r32 = (uint32_t)rj;
            if (lj > 1 && r32 % 10u == 0u) continue;  // j would have fewer digits
            const uint32_t j = rev_digits(r32, lj);
            if (j <= (uint32_t)K) mark(j);
        }
    }
}

// Row-tile sieve of the small primes.  grid = (tiles, triples).
__global__ void __launch_bounds__(kBlockTile)
small_tile_kernel(const SmallRec *__restrict__ rec, const uint32_t *__restrict__ counts, uint32_t cap,
                  int K, uint32_t *__restrict__ mask, size_t words_per_triple) {
    extern __shared__ uint32_t tile[];
    const int t = blockIdx.y;
    const uint32_t k0 = 1u + blockIdx.x * kTileRows;
    if (k0 > (uint32_t)K) return;
    const uint32_t k1 = min((uint32_t)K + 1u, k0 + kTileRows);
    const uint32_t rows = k1 - k0;
    const uint32_t bit_lo = (k0 - 1u) * (uint32_t)K;
    const uint32_t bit_hi = (k1 - 1u) * (uint32_t)K;
    const uint32_t w0 = bit_lo >> 5, w1 = (bit_hi - 1u) >> 5;
    const uint32_t nw = w1 - w0 + 1u;
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) tile[w] = 0u;
    __syncthreads();

    const uint32_t n_tiny = min(counts[0], cap / 2u), n_small = min(counts[1], cap / 2u);
    const SmallRec *rt = rec + (size_t)t * cap;
    const uint32_t bit_base = w0 << 5;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;

    // Tiny primes: one warp per (prime,row), lanes share the hits.
    for (uint32_t it = warp; it < n_tiny * rows; it += nwarps) {
        const SmallRec r = rt[it / rows];
        small_item(r, k0 + it % rows, K, lane, 32u, tile, bit_base);
    }
    // Other small primes: one thread per (prime,row).
    for (uint32_t it = threadIdx.x; it < n_small * rows; it += blockDim.x) {
        const SmallRec r = rt[n_tiny + it / rows];
        small_item(r, k0 + it % rows, K, 0u, 1u, tile, bit_base);
    }
    __syncthreads();
    uint32_t *g = mask + (size_t)t * words_per_triple + w0;
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
        const uint32_t v = tile[w];
        if (v) atomicOr(g + w, v);
    }
}

// Large primes (p >= S > K): each line meets every row at most once.  One
// thread per prime; incremental updates replace the multiplications.
__global__ void __launch_bounds__(kBlockLarge)
large_kernel(const uint32_t *__restrict__ primes, uint32_t n, uint32_t s_limit,
             const long long *__restrict__ abc, int K, uint32_t *__restrict__ mask,
             size_t words_per_triple) {
    const int t = blockIdx.y;
    const long long a = abc[3 * t], b = abc[3 * t + 1], c = abc[3 * t + 2];
    uint32_t *m = mask + (size_t)t * words_per_triple;
    const int maxd = ndigits(K);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = primes[i];
        if (p < s_limit) continue;
        Mod32 M;
        M.init(p);
        LineConsts lc;
        line_consts(M, a, b, c, lc);

        if (lc.flags & 1u)  // N form: j == AN - k BN (p > K: at most one j per k)
            line_hits(M, lc.an, lc.bn, 1u, (uint32_t)K, (uint32_t)K,
                      [&](uint32_t k, uint32_t j) { mark_global(m, K, k, j); });
        for (int lk = 1; lk <= maxd; lk++) {  // rev form, per digit class of k
            if (!(lc.flags & (1u << lk))) continue;
            const uint32_t lo = pow10i(lk - 1), hi = pow10i(lk) - 1u;
            // State of the four j classes in registers.  A class that is off
            // (no such digit count on the grid, or skipped by the reference's
            // rules) keeps value 0 and step 0: 0 never passes the hit test.
            uint32_t tv[4], st[4], on = 0u;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const bool c_on = (q + 1 <= maxd) && (lc.flags & (1u << (5 + q)));
                on |= c_on ? (1u << q) : 0u;
                st[q] = c_on ? lc.br[lk - 1][q] : 0u;
                tv[q] = c_on ? lc.ar[q] : 0u;
            }
            if (hi <= (uint32_t)K && lk >= 3) {
                // Long class (rev(k) takes up to 9999 values): per j class, a
                // lattice walk when rev(j) has >= 3 digits; otherwise iterate
                // the <= 99 values of rev(j): rev(k) == (AR - rev(j)) BR^-1,
                // BR^-1 = 10^(b-c+lk-lj) = BN * 10^(lk-lj).  (Not unrolled:
                // the walk is large and the instruction cache small.)
#pragma unroll 1
                for (int q = 0; q < 4; q++) {
                    if (!(on & (1u << q))) continue;
                    const int lj = q + 1;
                    const uint32_t ylim = pow10i(lj) - 1u;
                    if (lj >= 3) {
                        line_hits(M, lc.ar[q], st[q], 1u, hi, ylim, [&](uint32_t rk, uint32_t rj) {
                            if (rk % 10u != 0u && rj % 10u != 0u) {
                                const uint32_t j = rev_digits(rj, lj);
                                if (j <= (uint32_t)K) mark_global(m, K, rev_digits(rk, lk), j);
                            }
                        });
                    } else {
                        const uint32_t inv = M.mul(lc.bn, pow10i(lk - lj) % p);
                        uint32_t rk = M.mul(lc.ar[q], inv);  // rev(j) = 0
                        for (uint32_t rj = 1; rj <= ylim; rj++) {
                            rk = M.sub(rk, inv);
                            if (rk - 1u < hi && rk % 10u != 0u && (lj == 1 || rj % 10u != 0u)) {
                                const uint32_t j = rev_digits(rj, lj);
                                if (j <= (uint32_t)K) mark_global(m, K, rev_digits(rk, lk), j);
                            }
                        }
                    }
                }
            } else if (hi <= (uint32_t)K) {
                // short class (lk <= 2): walk rev(k) = 1 .. hi linearly
#pragma unroll
                for (int q = 0; q < 4; q++) tv[q] = M.sub(tv[q], st[q]);  // rk = 1
                for (uint32_t rk = 1; rk <= hi; rk++) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        if (tv[q] - 1u < pow10i(q + 1) - 1u) {  // 1 <= rev(j) < 10^(q+1)
                            const uint32_t rj = tv[q];
                            if ((lk == 1 || rk % 10u != 0u) && (q == 0 || rj % 10u != 0u)) {
                                const uint32_t j = rev_digits(rj, q + 1);
                                if (j <= (uint32_t)K) mark_global(m, K, rev_digits(rk, lk), j);
                            }
                        }
                        tv[q] = M.sub(tv[q], st[q]);
                    }
                }
            } else {
                // partial top class (K < 10^lk - 1): visit the k on the grid directly
                for (uint32_t k = lo; k <= (uint32_t)K; k++) {
                    const uint32_t rk = rev_digits(k, lk) % p;
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        if (!(on & (1u << q))) continue;
                        const uint32_t rj = M.sub(lc.ar[q], M.mul(rk, st[q]));
                        if (rj - 1u < pow10i(q + 1) - 1u && (q == 0 || rj % 10u != 0u)) {
                            const uint32_t j = rev_digits(rj, q + 1);
                            if (j <= (uint32_t)K) mark_global(m, K, k, j);
                        }
                    }
                }
            }
        }
    }
}

// Survivor compaction, pass 1: zero bits per 1024-bit chunk.
__global__ void surv_count_kernel(const uint32_t *__restrict__ mask, uint32_t nbits, uint32_t *chunk_cnt) {
    const uint32_t w = blockIdx.x * 32u + threadIdx.x;
    uint32_t c = 0;
    if (w * 32u < nbits) {
        uint32_t v = ~mask[w];
        const uint32_t rem = nbits - w * 32u;
        if (rem < 32u) v &= (1u << rem) - 1u;
        c = __popc(v);
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31u) == 0u) chunk_cnt[blockIdx.x] = c;
}

// Pass 2: exclusive scan of the chunk counts (single block).
__global__ void surv_scan_kernel(uint32_t *chunk_cnt, uint32_t n, uint32_t *total) {
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n ? chunk_cnt[i] : 0u;
        // block-wide inclusive scan (warp shuffles + smem)
        __shared__ uint32_t wsum[32];
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31u) >= (uint32_t)o) x += y;
        }
        if ((threadIdx.x & 31u) == 31u) wsum[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            uint32_t s = threadIdx.x < (blockDim.x >> 5) ? wsum[threadIdx.x] : 0u;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (threadIdx.x >= (uint32_t)o) s += y;
            }
            wsum[threadIdx.x] = s;
        }
        __syncthreads();
        const uint32_t wpre = (threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0u;
        const uint32_t incl = x + wpre;
        if (i < n) chunk_cnt[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// Pass 3: write (k << 16 | j) of every zero bit in k-major order.
__global__ void surv_write_kernel(const uint32_t *__restrict__ mask, uint32_t nbits, int K,
                                  const uint32_t *__restrict__ chunk_off, uint32_t *out, uint32_t cap) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t w = blockIdx.x * 32u + lane;
    uint32_t v = 0;
    if (w * 32u < nbits) {
        v = ~mask[w];
        const uint32_t rem = nbits - w * 32u;
        if (rem < 32u) v &= (1u << rem) - 1u;
    }
    const uint32_t c = __popc(v);
    uint32_t pre = c;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, pre, o);
        if (lane >= (uint32_t)o) pre += y;
    }
    uint32_t pos = chunk_off[blockIdx.x] + pre - c;
    while (v) {
        const uint32_t bit = __ffs(v) - 1u;
        v &= v - 1u;
        const uint32_t q = w * 32u + bit;
        const uint32_t k = q / (uint32_t)K + 1u, j = q % (uint32_t)K + 1u;
        if (pos < cap) out[pos] = (k << 16) | j;
        pos++;
    }
}

}  // namespace

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
        small_setup_kernel<<<g1, 128, 0, st>>>(s->d_tiny, s->d_small, s->d_counts, s->d_abc, n_abc, cap,
                                               s->d_rec);
        PFB_CUDA(cudaGetLastError());
        const uint32_t tiles = ((uint32_t)K + kTileRows - 1u) / kTileRows;
        const uint32_t max_rows = (uint32_t)K < (uint32_t)kTileRows ? (uint32_t)K : (uint32_t)kTileRows;
        const size_t smem = tile_smem_bytes(max_rows, K);
        dim3 g2(tiles, (unsigned)n_abc);
        small_tile_kernel<<<g2, kBlockTile, smem, st>>>(s->d_rec, s->d_counts, cap, K, d_mask, wpt);
        PFB_CUDA(cudaGetLastError());
    }
    if (s->n_primes) {
        int blocks = (int)((s->n_primes + kBlockLarge - 1) / kBlockLarge);
        dim3 g3((unsigned)blocks, (unsigned)n_abc);
        large_kernel<<<g3, kBlockLarge, 0, st>>>(s->d_primes, s->n_primes, s->s_limit, s->d_abc, K,
                                                 d_mask, wpt);
        PFB_CUDA(cudaGetLastError());
    }
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

constexpr uint32_t kNoAllocListCap = 10000u / 2u + 2u;  // small primes (< 10000) per list

struct NoAllocScratch {
    uint32_t counts[2];
    uint32_t pad0[62];
    long long abc[4];
    uint32_t tiny[kNoAllocListCap];
    uint32_t small[kNoAllocListCap];
    SmallRec rec[2 * kNoAllocListCap];
};

// 1.16 MB: the scratch of one triple at any K <= 9999.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

__global__ void noalloc_begin_kernel(NoAllocScratch *sc, long long a, long long b, long long c) {
    sc->counts[0] = 0u;
    sc->counts[1] = 0u;
    sc->abc[0] = a;
    sc->abc[1] = b;
    sc->abc[2] = c;
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
    noalloc_begin_kernel<<<1, 1, 0, st>>>(sc, a, b, c);
    PFB_CUDA(cudaGetLastError());
    const uint32_t lim = small_limit(K);
    const uint32_t cap = kNoAllocListCap;
    if (n_primes) {
        const int blocks = (int)std::min<uint32_t>((n_primes + 255u) / 256u, (uint32_t)sms * 16u);
        split_kernel<<<blocks, 256, 0, st>>>(d_primes, n_primes, lim, cap, sc->tiny, sc->small, sc->counts);
        PFB_CUDA(cudaGetLastError());
        // record stride 2*cap: tiny then small; the kernels read the counts on the device
        dim3 g1((2u * cap + 127u) / 128u, 1u);
        small_setup_kernel<<<g1, 128, 0, st>>>(sc->tiny, sc->small, sc->counts, sc->abc, 1, 2u * cap, sc->rec);
        PFB_CUDA(cudaGetLastError());
        const uint32_t tiles = ((uint32_t)K + kTileRows - 1u) / kTileRows;
        const uint32_t rows = (uint32_t)K < (uint32_t)kTileRows ? (uint32_t)K : (uint32_t)kTileRows;
        small_tile_kernel<<<dim3(tiles, 1u), kBlockTile, tile_smem_bytes(rows, K), st>>>(sc->rec, sc->counts,
                                                                                         2u * cap, K, d_mask, wpt);
        PFB_CUDA(cudaGetLastError());
        const int lb = (int)((n_primes + kBlockLarge - 1) / kBlockLarge);
        large_kernel<<<dim3((unsigned)lb, 1u), kBlockLarge, 0, st>>>(d_primes, n_primes, lim, sc->abc, K, d_mask,
                                                                    wpt);
        PFB_CUDA(cudaGetLastError());
    }
    return PFB_OK;
}
