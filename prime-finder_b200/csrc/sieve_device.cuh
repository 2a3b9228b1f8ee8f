// Device side of the Phase-1 sieve (sieve.cu): launch constants, the line
// coefficients, the lattice walk and every kernel.  Included by sieve.cu
// only; kept apart from the host code so that the kernels can also be
// compiled for the host and run on CPU threads in the tests.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

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

// Coefficients of the two lines of a prime p coprime to 10 (D the digit
// count of K, X = 10^D - 1):
//
//   N form    j == an - k bn (mod p),  an = (10^a - 1) 10^-c,  bn = 10^(b-c)
//   rev form  y == ar - x br (mod p),  ar = (10^a - 1) 10^(c+D-a),  br = 10^(c-b)
//
// The rev form of trial_div_cpu.c:54-101 has one congruence per digit class
// (lk, lj) of (k, j): rev(j) == (10^a - 1) 10^(c+lj-a) - rev(k) 10^(c-b+lj-lk).
// Multiplied by 10^(D-lj) it is the single congruence above at
// x = rev(k) 10^(D-lk), y = rev(j) 10^(D-lj), both in [1, X]; as 10 is
// invertible mod p the two are equivalent.  Conversely every solution (x, y)
// in [1, X]^2 is the point of exactly one class: x written with D digits
// (leading zeros allowed) and reversed is k, whose digit count is lk (k never
// starts with 0), likewise for y and j.  One line over x, y in [1, X] thus
// holds the hits of all D x D classes.  The reference uses a class of lk
// digits only when a - b - lk >= 0 (of lj digits: a - c - lj >= 0,
// trial_div_cpu.c:59-66, 78-84), i.e. when k < 10^(a-b) (j < 10^(a-c)):
// class_max.  The N form is always used for such p (trial_div_cpu.c:40-52).
struct LineCoeffs {
    uint32_t an, bn, ar, br;
};

__device__ void line_coeffs(const Mod32 &M, long long a, long long b, long long c, int D, LineCoeffs &s) {
    const uint32_t p = M.p;
    const uint32_t d = p % 10u;
    const uint32_t t = d == 1 ? 9u : d == 3 ? 3u : d == 7 ? 7u : 1u;
    const uint32_t inv10 = (uint32_t)(((unsigned long long)p * t + 1ull) / 10ull);
    const uint32_t ten = 10u % p;
    // 10^e for any integer e
    auto pw = [&](long long e) -> uint32_t {
        return e >= 0 ? M.pow(ten, (unsigned long long)e) : M.pow(inv10, (unsigned long long)(-e));
    };
    const uint32_t ram1 = M.sub(pw(a), 1u % p);
    s.an = M.mul(ram1, pw(-c));
    s.bn = pw(b - c);
    s.ar = M.mul(ram1, pw(c + D - a));
    s.br = pw(c - b);
}

// Largest k (or j) of a class the reference uses, e = a - b (or a - c):
// min(K, 10^min(e, D) - 1), 0 when no class is used.
__device__ __forceinline__ uint32_t class_max(long long e, int D, int K) {
    if (e < 1) return 0u;
    const uint32_t m = pow10i(e < D ? (int)e : D) - 1u;
    return m < (uint32_t)K ? m : (uint32_t)K;
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
// the tile kernel: p, its Barrett constant and the coefficients of its two
// lines (line_coeffs).  legacy = 1 for a p that shares a factor with 10 (5,
// and 2 when listed): the tile kernel then takes the reference's per-class
// congruences (line_consts), which the one-line form cannot merge.
struct SmallRec {
    uint32_t p;
    uint32_t m_lo, m_hi;
    uint32_t an, bn, ar, br;
    uint32_t legacy;
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

// The descent keeps, per level, the multiplier a and the interval start L
// packed in one 64-bit word, and the reciprocal of a (one 64-bit store and
// load each per level); the level's modulus is the previous level's
// multiplier (p at level 0), which the way back already holds.
__device__ __noinline__ uint32_t first_hit(uint32_t c, uint32_t g, uint32_t p, uint32_t Y) {
    if (c < Y) return 0u;
    uint32_t a = g, m = p, L = p - c, R = p - c + Y - 1u;
    unsigned long long st[34];
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
        st[d] = ((unsigned long long)L << 32) | a;
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
    unsigned long long cur = d ? st[d - 1] : 0ull;
    while (d > 0) {
        d--;
        const uint32_t ad = (uint32_t)cur, ld = (uint32_t)(cur >> 32);
        const unsigned long long prev = d ? st[d - 1] : (unsigned long long)p;
        const uint32_t md = (uint32_t)prev;
        x = (uint32_t)quot64((unsigned long long)x * md + ld + ad - 1u, ad, sr[d]);  // ceil
        cur = prev;
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

// Calls visit(x0 + t, i + 1) for every t in [0, x1 - x0] with
// i = (c0 + g t) mod p < Y; i_of(t) computes (c0 + g t) mod p.  Requires
// 1 <= Y < p, g != 0, x1 - x0 < p.
template <class IOf, class Visit>
__device__ __forceinline__ void walk_hits(uint32_t c0, uint32_t g, uint32_t p, uint32_t x0, uint32_t x1, uint32_t Y,
                                          IOf i_of, Visit visit) {
    unsigned long long t = first_hit(c0, g, p, Y);
    const unsigned long long span = (unsigned long long)(x1 - x0);
    if (t > span) return;
    const FKBasis fb = fk_reduce(g, p, Y);
    uint32_t i = i_of((uint32_t)t);
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

// Montgomery arithmetic for an odd modulus p < 2^32, R = 2^32: mul(a, b) =
// a b R^-1 mod p for a, b < p.  m = lo(a b) p^-1 mod R makes a b - m p a
// multiple of R, so the result is hi(a b) - hi(m p) (+ p): two mul.hi, two
// mul.lo, no 64-bit sums.
struct Mont32 {
    uint32_t p, pinv;  // pinv = p^-1 mod 2^32

    __device__ __forceinline__ void init(uint32_t p_) {
        p = p_;
        uint32_t x = p_;  // p x == 1 (mod 2^3) for odd p; each step doubles the bits
        x *= 2u - p_ * x;
        x *= 2u - p_ * x;
        x *= 2u - p_ * x;
        x *= 2u - p_ * x;
        pinv = x;
    }
    __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const {
        const uint32_t hi = __umulhi(a, b), m = (a * b) * pinv, h = __umulhi(m, p);
        return hi >= h ? hi - h : hi - h + p;
    }
    __device__ __forceinline__ uint32_t add(uint32_t a, uint32_t b) const {
        const uint32_t s = a + b;
        return (s < a || s >= p) ? s - p : s;
    }
    __device__ __forceinline__ uint32_t sub(uint32_t a, uint32_t b) const { return a >= b ? a - b : a - b + p; }
};

// Calls visit(x, y) for every x in [x0, x1] with y = (A - B x) mod p in
// [1, Y]; requires 1 <= Y < p, B != 0 (mod p), x0 <= x1 < p.  Bm = B R mod
// p: B x0 mod p is mul(Bm, x0) and g t mod p is mul(gm, t), so no 64-bit
// value is reduced.
template <class Visit>
__device__ __forceinline__ void line_hits_m(const Mont32 &M, uint32_t A, uint32_t B, uint32_t Bm, uint32_t x0,
                                            uint32_t x1, uint32_t Y, Visit visit) {
    const uint32_t p = M.p, g = p - B, gm = p - Bm;
    const uint32_t c0 = M.sub(M.sub(A, 1u), M.mul(Bm, x0));
    walk_hits(c0, g, p, x0, x1, Y, [&](uint32_t t) { return M.add(M.mul(gm, t), c0); }, visit);
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

// split_kernel for lists of fixed capacity (the allocation-free entry
// point): a value is listed once however often the prime list repeats it
// (seen: a bitmap over [0, s_limit), cleared by the caller), and even values,
// never prime above 2 (2 eliminates nothing: N and rev(N) are odd), are
// skipped.  At most the odd values in [3, s_limit) are listed, so lists of
// s_limit/2 + 2 entries cannot overflow, whatever the input.
__global__ void split_unique_kernel(const uint32_t *__restrict__ primes, uint32_t n, uint32_t s_limit,
                                    uint32_t *seen, uint32_t *tiny, uint32_t *small, uint32_t *counts) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = primes[i];
        if (p < 3u || p >= s_limit || !(p & 1u)) continue;
        const uint32_t bit = 1u << (p & 31u);
        if (atomicOr(&seen[p >> 5], bit) & bit) continue;
        if (p < kTinyLimit) tiny[atomicAdd(&counts[0], 1u)] = p;
        else small[atomicAdd(&counts[1], 1u)] = p;
    }
}

// Set-up of the small-prime records for every triple: rec[t * cap + i];
// cap = 2 * capacity of each list.
__global__ void small_setup_kernel(const uint32_t *__restrict__ tiny, const uint32_t *__restrict__ small,
                                   const uint32_t *__restrict__ counts, const long long *__restrict__ abc,
                                   int n_abc, int K, uint32_t cap, SmallRec *__restrict__ rec) {
    const uint32_t n_tiny = min(counts[0], cap / 2u), n_small = min(counts[1], cap / 2u);
    const uint32_t n = n_tiny + n_small;
    const int t = blockIdx.y;
    if (t >= n_abc) return;
    const int D = ndigits(K);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = i < n_tiny ? tiny[i] : small[i - n_tiny];
        Mod32 M;
        M.init(p);
        SmallRec r;
        r.p = p;
        r.m_lo = (uint32_t)M.m;
        r.m_hi = (uint32_t)(M.m >> 32);
        r.legacy = (p % 2u == 0u || p % 5u == 0u) ? 1u : 0u;
        LineCoeffs lc{0u, 0u, 0u, 0u};
        if (!r.legacy) line_coeffs(M, abc[3 * t], abc[3 * t + 1], abc[3 * t + 2], D, lc);
        r.an = lc.an;
        r.bn = lc.bn;
        r.ar = lc.ar;
        r.br = lc.br;
        rec[(size_t)t * cap + i] = r;
    }
}

// Marks of one (prime,row) item in the tile.  Lanes lane0, lane0+step, ...
// of the hit sequences are handled by this thread (step = 32 for warp items,
// 1 for thread items).  Row k: the N-form hits j == an - k bn (mod p), and
// the rev-form hits y == ar - rev_D(k) br (mod p), y in [1, X], j = rev_D(y),
// of the classes in use (k <= kmax, j <= jmax).
template <int D>
__device__ __forceinline__ void small_item(const SmallRec &r, uint32_t k, int K, uint32_t kmax, uint32_t jmax,
                                           uint32_t lane0, uint32_t step, uint32_t *tile, uint32_t bit_base) {
    constexpr uint32_t X = D == 1 ? 9u : D == 2 ? 99u : D == 3 ? 999u : 9999u;
    Mod32 M;
    M.p = r.p;
    M.m = ((unsigned long long)r.m_hi << 32) | r.m_lo;
    const uint32_t p = r.p;
    const uint32_t row = (k - 1u) * (uint32_t)K - bit_base;
    auto mark = [&](uint32_t j) {
        const uint32_t q = row + (j - 1u);
        atomicOr(tile + (q >> 5), 1u << (q & 31u));
    };
    uint32_t j0 = M.sub(r.an, M.mul(k % p, r.bn));
    if (j0 == 0) j0 = p;
    for (uint32_t j = j0 + lane0 * p; j <= (uint32_t)K; j += step * p) mark(j);
    if (k > kmax) return;
    uint32_t y0 = M.sub(r.ar, M.mul(rev_digits(k, D) % p, r.br));
    if (y0 == 0) y0 = p;
    for (uint32_t y = y0 + lane0 * p; y <= X; y += step * p) {
        const uint32_t j = rev_digits(y, D);
        if (j <= jmax) mark(j);
    }
}

// The same for a p that shares a factor with 10, on the reference's
// per-class congruences (line_consts).
__device__ void small_item_legacy(const SmallRec &r, const long long *abc, uint32_t k, int K, uint32_t lane0,
                                  uint32_t step, uint32_t *tile, uint32_t bit_base) {
    Mod32 M;
    M.p = r.p;
    M.m = ((unsigned long long)r.m_hi << 32) | r.m_lo;
    const uint32_t p = r.p;
    LineConsts lc;
    line_consts(M, abc[0], abc[1], abc[2], lc);
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

template <int D>
__device__ __forceinline__ void small_rows(const SmallRec *rt, uint32_t n_tiny, uint32_t n_small,
                                           const long long *abc, uint32_t k0, uint32_t rows, int K,
                                           uint32_t *tile, uint32_t bit_base) {
    const uint32_t kmax = class_max(abc[0] - abc[1], D, K), jmax = class_max(abc[0] - abc[2], D, K);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    // Tiny primes: one warp per (prime,row), lanes share the hits.
    for (uint32_t it = warp; it < n_tiny * rows; it += nwarps) {
        const SmallRec r = rt[it / rows];
        const uint32_t k = k0 + it % rows;
        if (r.legacy) small_item_legacy(r, abc, k, K, lane, 32u, tile, bit_base);
        else small_item<D>(r, k, K, kmax, jmax, lane, 32u, tile, bit_base);
    }
    // Other small primes: one thread per (prime,row).
    for (uint32_t it = threadIdx.x; it < n_small * rows; it += blockDim.x) {
        const SmallRec r = rt[n_tiny + it / rows];
        const uint32_t k = k0 + it % rows;
        if (r.legacy) small_item_legacy(r, abc, k, K, 0u, 1u, tile, bit_base);
        else small_item<D>(r, k, K, kmax, jmax, 0u, 1u, tile, bit_base);
    }
}

// Row-tile sieve of the small primes.  grid = (tiles, triples).
__global__ void __launch_bounds__(kBlockTile)
small_tile_kernel(const SmallRec *__restrict__ rec, const uint32_t *__restrict__ counts, uint32_t cap,
                  const long long *__restrict__ abc, int K, uint32_t *__restrict__ mask,
                  size_t words_per_triple) {
    PFB_DYNAMIC_SMEM(uint32_t, tile);
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
    const long long *tabc = abc + 3 * t;
    switch (ndigits(K)) {
    case 1: small_rows<1>(rt, n_tiny, n_small, tabc, k0, rows, K, tile, bit_base); break;
    case 2: small_rows<2>(rt, n_tiny, n_small, tabc, k0, rows, K, tile, bit_base); break;
    case 3: small_rows<3>(rt, n_tiny, n_small, tabc, k0, rows, K, tile, bit_base); break;
    default: small_rows<4>(rt, n_tiny, n_small, tabc, k0, rows, K, tile, bit_base); break;
    }
    __syncthreads();
    uint32_t *g = mask + (size_t)t * words_per_triple + w0;
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
        const uint32_t v = tile[w];
        if (v) atomicOr(g + w, v);
    }
}

// A prime of the large-prime kernels: at least the small limit and above
// 10^D - 1, and coprime to 10 (anything else in the list is not a prime).
__device__ __forceinline__ bool large_prime(uint32_t p, uint32_t lo, uint32_t hi, uint32_t X) {
    return p >= lo && p < hi && p > X && (p & 1u) && p % 5u != 0u;
}

// The line_coeffs coefficients, plain (an, bn, ar, br) and bn, br in
// Montgomery form (bnm, brm).  The five powers 10^a, 10^-c, 10^(b-c),
// 10^(c+D-a), 10^(c-b) come from one right-to-left binary exponentiation
// over the exponents' bits: the squarings of 10 and of 10^-1 are shared,
// each power multiplies in the square of its bits.  The exponents are the
// triple's, the same in every thread, so the branches are uniform.
struct LineCoeffsM {
    uint32_t an, bn, ar, br, bnm, brm;
};

__device__ void line_coeffs_m(const Mont32 &M, long long a, long long b, long long c, int D, LineCoeffsM &s) {
    const uint32_t p = M.p;
    const uint32_t one = (0u - p) % p;  // R mod p
    // 10 R mod p (doublings), R / 10 mod p = (R + k p) / 10 with R + k p == 0 (mod 10)
    const uint32_t r2 = M.add(one, one), r4 = M.add(r2, r2), r8 = M.add(r4, r4);
    uint32_t x10 = M.add(r8, r2);
    const uint32_t pd = p % 10u, pi = pd == 1 ? 1u : pd == 3 ? 7u : pd == 7 ? 3u : 9u;  // p^-1 mod 10
    const uint32_t k = ((10u - one % 10u) % 10u) * pi % 10u;
    uint32_t xi = (uint32_t)(((unsigned long long)one + (unsigned long long)k * p) / 10ull);
    const long long e[5] = {a, -c, b - c, c + D - a, c - b};
    unsigned long long m[5];
    uint32_t acc[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
        m[q] = (unsigned long long)(e[q] < 0 ? -e[q] : e[q]);
        acc[q] = one;
    }
    for (;;) {
        bool more = false;
#pragma unroll
        for (int q = 0; q < 5; q++) {
            if (m[q] & 1ull) acc[q] = M.mul(acc[q], e[q] < 0 ? xi : x10);
            m[q] >>= 1;
            more |= m[q] != 0ull;
        }
        if (!more) break;
        x10 = M.mul(x10, x10);
        xi = M.mul(xi, xi);
    }
    const uint32_t ram1 = M.sub(acc[0], one);  // (10^a - 1) R
    s.bnm = acc[2];
    s.brm = acc[4];
    s.an = M.mul(M.mul(ram1, acc[1]), 1u);
    s.bn = M.mul(acc[2], 1u);
    s.ar = M.mul(M.mul(ram1, acc[3]), 1u);
    s.br = M.mul(acc[4], 1u);
}

// Hits of one prime on x in [x0, x1] of both lines (x1 <= K on the N line,
// <= X on the rev line; an empty range when x0 > x1).
template <int D>
__device__ __forceinline__ void large_lines(const Mont32 &M, const LineCoeffsM &lc, uint32_t nx0, uint32_t nx1,
                                            uint32_t rx0, uint32_t rx1, uint32_t kmax, uint32_t jmax, int K,
                                            uint32_t *m) {
    constexpr uint32_t X = D == 1 ? 9u : D == 2 ? 99u : D == 3 ? 999u : 9999u;
    if (nx0 <= nx1)  // N form (trial_div_cpu.c:40-52): at most one j per k
        line_hits_m(M, lc.an, lc.bn, lc.bnm, nx0, nx1, (uint32_t)K,
                    [&](uint32_t k, uint32_t j) { mark_global(m, K, k, j); });
    if (rx0 <= rx1 && kmax && jmax)
        line_hits_m(M, lc.ar, lc.br, lc.brm, rx0, rx1, X, [&](uint32_t x, uint32_t y) {
            const uint32_t k = rev_digits(x, D), j = rev_digits(y, D);
            if (k <= kmax && j <= jmax) mark_global(m, K, k, j);
        });
}

// Primes in [p_med, inf): one thread per prime, whole lines.  At most about
// 2 K^2 / p_med hits per thread.
template <int D>
__global__ void __launch_bounds__(kBlockLarge)
large_kernel(const uint32_t *__restrict__ primes, uint32_t n, uint32_t p_med,
             const long long *__restrict__ abc, int K, uint32_t *__restrict__ mask,
             size_t words_per_triple) {
    constexpr uint32_t X = D == 1 ? 9u : D == 2 ? 99u : D == 3 ? 999u : 9999u;
    const int t = blockIdx.y;
    const long long a = abc[3 * t], b = abc[3 * t + 1], c = abc[3 * t + 2];
    uint32_t *m = mask + (size_t)t * words_per_triple;
    const uint32_t kmax = class_max(a - b, D, K), jmax = class_max(a - c, D, K);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = primes[i];
        if (!large_prime(p, p_med, 0xFFFFFFFFu, X)) continue;
        Mont32 M;
        M.init(p);
        LineCoeffsM lc;
        line_coeffs_m(M, a, b, c, D, lc);
        large_lines<D>(M, lc, 1u, (uint32_t)K, 1u, X, kmax, jmax, K, m);
    }
}

// Primes in [s_limit, p_med), the ones with the most hits: a warp per
// prime, lane l walking the l-th 32nd of each line's x range, so that no
// single thread carries the ~2 K^2 / p hits of a small large prime.  Warp w
// of W loads the list entries w + l W (lane l), then w + (32 + l) W, ...; on
// a sorted list that hands every warp primes from across the whole range.
// A lane that loaded a prime of the range sets up its lines, then the warp
// walks the primes of the batch one after another, their constants
// broadcast from the lane that holds them.
template <int D>
__global__ void __launch_bounds__(kBlockLarge)
medium_kernel(const uint32_t *__restrict__ primes, uint32_t n, uint32_t s_limit, uint32_t p_med,
              const long long *__restrict__ abc, int K, uint32_t *__restrict__ mask,
              size_t words_per_triple) {
    constexpr uint32_t X = D == 1 ? 9u : D == 2 ? 99u : D == 3 ? 999u : 9999u;
    const int t = blockIdx.y;
    const long long a = abc[3 * t], b = abc[3 * t + 1], c = abc[3 * t + 2];
    uint32_t *m = mask + (size_t)t * words_per_triple;
    const uint32_t kmax = class_max(a - b, D, K), jmax = class_max(a - c, D, K);
    const uint32_t lane = threadIdx.x & 31u;
    const size_t W = (size_t)gridDim.x * (blockDim.x >> 5);
    const size_t w = (size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t nseg = ((uint32_t)K + 31u) / 32u, rseg = (X + 31u) / 32u;
    const uint32_t nx0 = 1u + lane * nseg, rx0 = 1u + lane * rseg;
    const uint32_t nx1 = min((uint32_t)K, nx0 + nseg - 1u), rx1 = min(X, rx0 + rseg - 1u);
    for (size_t base = w; base < n; base += 32u * W) {
        const size_t e = base + lane * W;
        const uint32_t p = e < n ? primes[e] : 0u;
        const bool mine = large_prime(p, s_limit, p_med, X);
        unsigned todo = __ballot_sync(0xFFFFFFFFu, mine);
        Mont32 M;
        M.p = 0u;
        M.pinv = 0u;
        LineCoeffsM lc{0u, 0u, 0u, 0u, 0u, 0u};
        if (mine) {
            M.init(p);
            line_coeffs_m(M, a, b, c, D, lc);
        }
        while (todo) {
            const int src = __ffs((int)todo) - 1;
            todo &= todo - 1u;
            Mont32 Ms;
            Ms.p = __shfl_sync(0xFFFFFFFFu, M.p, src);
            Ms.pinv = __shfl_sync(0xFFFFFFFFu, M.pinv, src);
            LineCoeffsM ls;
            ls.an = __shfl_sync(0xFFFFFFFFu, lc.an, src);
            ls.bn = __shfl_sync(0xFFFFFFFFu, lc.bn, src);
            ls.ar = __shfl_sync(0xFFFFFFFFu, lc.ar, src);
            ls.br = __shfl_sync(0xFFFFFFFFu, lc.br, src);
            ls.bnm = __shfl_sync(0xFFFFFFFFu, lc.bnm, src);
            ls.brm = __shfl_sync(0xFFFFFFFFu, lc.brm, src);
            large_lines<D>(Ms, ls, nx0, nx1, rx0, rx1, kmax, jmax, K, m);
        }
    }
}

// Bottom of the large-prime kernel's range: primes below it have more than
// about 12 000 hits per thread and go to the medium kernel.  Measured on one
// K = 9999 triple (medium + large): 3.06 ms with no medium kernel, 2.83 ms
// with the limit at 12 000 to 16 384, 3.01 ms at 2^18.
inline uint32_t medium_limit(int K, uint32_t s_limit) {
    const unsigned long long X = pow10i(ndigits(K)) - 1u;
    const unsigned long long h = ((unsigned long long)K * (unsigned long long)K + X * X) / 12288ull;
    const uint32_t v = h < (1ull << 18) ? (uint32_t)h : (1u << 18);
    return v > s_limit ? v : s_limit;
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
