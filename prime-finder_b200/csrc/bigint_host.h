// Host-side multi-precision helpers for the Miller-Rabin set-up.
//
// The reference does this set-up with GMP on the host (Barrett's mu,
// barrett.cu:29-107; Montgomery's N', montgomery.cu:30-45; residues of the
// witness, miller_rabin_runner.cu:315-325).  This engine needs, per modulus
// N and Montgomery radix R = 2^(22*H):
//   * N' = -N^-1 mod R                 (Hensel lifting)
//   * R mod N                          (Knuth's long division, TAOCP 4.3.1 D)
//   * N - 1 = 2^s * d                  (bit scan)
// Numbers are little-endian vectors of 64-bit words.
#pragma once
#include <stdint.h>

#include <algorithm>
#include <vector>

namespace pfb {
namespace big {

using Words = std::vector<uint64_t>;

inline void trim(Words &a) {
    while (!a.empty() && a.back() == 0) a.pop_back();
}

inline size_t bit_length(const Words &a) {
    for (size_t i = a.size(); i-- > 0;)
        if (a[i]) return i * 64 + (64 - __builtin_clzll(a[i]));
    return 0;
}

inline bool test_bit(const Words &a, size_t i) {
    return (i / 64 < a.size()) && ((a[i / 64] >> (i % 64)) & 1ull);
}

inline Words from_u16(const uint16_t *l, size_t n) {
    Words w((n + 3) / 4, 0);
    for (size_t i = 0; i < n; i++) w[i / 4] |= (uint64_t)l[i] << (16 * (i % 4));
    trim(w);
    return w;
}

inline void to_u16(const Words &a, uint16_t *out, size_t n) {
    for (size_t i = 0; i < n; i++) out[i] = (i / 4 < a.size()) ? (uint16_t)(a[i / 4] >> (16 * (i % 4))) : 0;
}

// Little-endian `bits`-bit limbs (bits <= 32), exactly n of them.
inline void to_limbs(const Words &a, unsigned bits, uint32_t *out, size_t n) {
    const uint64_t mask = (1ull << bits) - 1ull;
    for (size_t i = 0; i < n; i++) {
        const size_t bit = i * bits, wi = bit / 64, sh = bit % 64;
        uint64_t v = 0;
        if (wi < a.size()) {
            v = a[wi] >> sh;
            if (sh + bits > 64 && wi + 1 < a.size()) v |= a[wi + 1] << (64 - sh);
        }
        out[i] = (uint32_t)(v & mask);
    }
}

inline Words from_limbs(const uint32_t *l, unsigned bits, size_t n) {
    Words w((n * bits + 63) / 64 + 1, 0);
    for (size_t i = 0; i < n; i++) {
        const size_t bit = i * bits, wi = bit / 64, sh = bit % 64;
        w[wi] |= (uint64_t)l[i] << sh;
        if (sh + bits > 64) w[wi + 1] |= (uint64_t)l[i] >> (64 - sh);
    }
    trim(w);
    return w;
}

inline int cmp(const Words &a, const Words &b) {
    if (a.size() != b.size()) return a.size() < b.size() ? -1 : 1;
    for (size_t i = a.size(); i-- > 0;)
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
}

inline Words sub_small(Words a, uint64_t s) {
    for (size_t i = 0; i < a.size() && s; i++) {
        const uint64_t v = a[i];
        a[i] = v - s;
        s = (v < s) ? 1 : 0;
    }
    trim(a);
    return a;
}

inline Words shr(const Words &a, size_t s) {
    const size_t ws = s / 64, bs = s % 64;
    if (ws >= a.size()) return Words();
    Words r(a.size() - ws, 0);
    for (size_t i = 0; i < r.size(); i++) {
        uint64_t v = a[i + ws] >> bs;
        if (bs && i + ws + 1 < a.size()) v |= a[i + ws + 1] << (64 - bs);
        r[i] = v;
    }
    trim(r);
    return r;
}

// (a * b) mod 2^(64*k), schoolbook, truncated.
inline Words mullo(const Words &a, const Words &b, size_t k) {
    Words r(k, 0);
    for (size_t i = 0; i < a.size() && i < k; i++) {
        unsigned __int128 carry = 0;
        const uint64_t ai = a[i];
        if (!ai) continue;
        for (size_t j = 0; j < b.size() && i + j < k; j++) {
            unsigned __int128 t = (unsigned __int128)ai * b[j] + r[i + j] + carry;
            r[i + j] = (uint64_t)t;
            carry = t >> 64;
        }
        for (size_t j = i + b.size(); j < k && carry; j++) {
            unsigned __int128 t = (unsigned __int128)r[j] + carry;
            r[j] = (uint64_t)t;
            carry = t >> 64;
        }
    }
    return r;
}

// -N^-1 mod 2^bits for odd N (Hensel / Newton: x <- x*(2 - N*x)).
inline Words neg_inv_pow2(const Words &N, size_t bits) {
    uint64_t x0 = N[0];  // N*N == 1 mod 8 for odd N
    for (int i = 0; i < 6; i++) x0 *= 2 - N[0] * x0;
    Words x(1, x0);
    size_t k = 1;
    const size_t kmax = (bits + 63) / 64;
    while (k < kmax) {
        k = std::min(2 * k, kmax);
        Words nx = mullo(N, x, k);           // N*x = 1 + e
        // 2 - N*x  (mod 2^(64k))
        Words t(k, 0);
        unsigned __int128 borrow = 0;
        for (size_t i = 0; i < k; i++) {
            const uint64_t two = (i == 0) ? 2 : 0;
            const uint64_t v = (i < nx.size()) ? nx[i] : 0;
            unsigned __int128 d = (unsigned __int128)two - v - (uint64_t)borrow;
            t[i] = (uint64_t)d;
            borrow = (d >> 64) ? 1 : 0;
        }
        x = mullo(x, t, k);
    }
    // negate mod 2^(64*kmax), then truncate to `bits`
    Words r(kmax, 0);
    unsigned __int128 carry = 1;
    for (size_t i = 0; i < kmax; i++) {
        unsigned __int128 v = (unsigned __int128)(uint64_t)(~(i < x.size() ? x[i] : 0ull)) + carry;
        r[i] = (uint64_t)v;
        carry = v >> 64;
    }
    if (bits % 64) r[kmax - 1] &= (1ull << (bits % 64)) - 1ull;
    trim(r);
    return r;
}

// Quotient and remainder of U / V (V > 0) by Knuth's algorithm D on 32-bit
// digits (TAOCP vol. 2, 4.3.1).
inline void divmod(const Words &U, const Words &V, Words *quot, Words *rem) {
    auto digits = [](const Words &a) {
        std::vector<uint32_t> d;
        for (uint64_t w : a) {
            d.push_back((uint32_t)w);
            d.push_back((uint32_t)(w >> 32));
        }
        while (!d.empty() && d.back() == 0) d.pop_back();
        return d;
    };
    auto words = [](const std::vector<uint32_t> &d) {
        Words w((d.size() + 1) / 2, 0);
        for (size_t i = 0; i < d.size(); i++) w[i / 2] |= (uint64_t)d[i] << (32 * (i % 2));
        trim(w);
        return w;
    };
    const std::vector<uint32_t> v = digits(V), u = digits(U);
    const size_t n = v.size();
    if (u.size() < n || cmp(U, V) < 0) {
        if (quot) *quot = Words();
        if (rem) {
            *rem = U;
            trim(*rem);
        }
        return;
    }
    const size_t m = u.size() - n;
    std::vector<uint32_t> q(m + 1, 0);
    if (n == 1) {
        uint64_t r = 0;
        for (size_t i = u.size(); i-- > 0;) {
            const uint64_t cur = (r << 32) | u[i];
            if (i <= m) q[i] = (uint32_t)(cur / v[0]);
            r = cur % v[0];
        }
        if (quot) *quot = words(q);
        if (rem) *rem = r ? Words(1, r) : Words();
        return;
    }
    const int s = __builtin_clz(v[n - 1]);
    std::vector<uint32_t> vn(n), un(u.size() + 1);
    for (size_t i = n - 1; i > 0; i--) vn[i] = (v[i] << s) | (s ? (uint32_t)((uint64_t)v[i - 1] >> (32 - s)) : 0u);
    vn[0] = v[0] << s;
    un[u.size()] = s ? (uint32_t)((uint64_t)u[u.size() - 1] >> (32 - s)) : 0u;
    for (size_t i = u.size() - 1; i > 0; i--) un[i] = (u[i] << s) | (s ? (uint32_t)((uint64_t)u[i - 1] >> (32 - s)) : 0u);
    un[0] = u[0] << s;
    const uint64_t b = 1ull << 32;
    for (size_t jj = m + 1; jj-- > 0;) {
        const size_t j = jj;
        const uint64_t num = ((uint64_t)un[j + n] << 32) | un[j + n - 1];
        uint64_t qhat = num / vn[n - 1];
        uint64_t rhat = num - qhat * vn[n - 1];
        while (qhat >= b || qhat * vn[n - 2] > ((rhat << 32) | un[j + n - 2])) {
            qhat--;
            rhat += vn[n - 1];
            if (rhat >= b) break;
        }
        int64_t borrow = 0;
        uint64_t carry = 0;
        for (size_t i = 0; i < n; i++) {
            const uint64_t p = qhat * vn[i] + carry;
            carry = p >> 32;
            const int64_t t = (int64_t)un[i + j] - (int64_t)(uint32_t)p - borrow;
            un[i + j] = (uint32_t)t;
            borrow = (t < 0) ? 1 : 0;
        }
        const int64_t t = (int64_t)un[j + n] - (int64_t)carry - borrow;
        un[j + n] = (uint32_t)t;
        if (t < 0) {  // add back
            qhat--;
            uint64_t c = 0;
            for (size_t i = 0; i < n; i++) {
                const uint64_t sum = (uint64_t)un[i + j] + vn[i] + c;
                un[i + j] = (uint32_t)sum;
                c = sum >> 32;
            }
            un[j + n] += (uint32_t)c;
        }
        q[j] = (uint32_t)qhat;
    }
    if (quot) *quot = words(q);
    if (rem) {
        std::vector<uint32_t> r(n);
        for (size_t i = 0; i < n; i++)
            r[i] = (un[i] >> s) | (s ? (uint32_t)((uint64_t)un[i + 1] << (32 - s)) : 0u);
        *rem = words(r);
    }
}

// 2^e mod N (N > 1).
inline Words pow2_mod(size_t e, const Words &N) {
    Words u(e / 64 + 1, 0);
    u[e / 64] = 1ull << (e % 64);
    Words r;
    divmod(u, N, nullptr, &r);
    return r;
}

// a mod m for 0 < m < 2^32.
inline uint32_t mod_small(const Words &a, uint32_t m) {
    unsigned __int128 r = 0;
    for (size_t i = a.size(); i-- > 0;) r = ((r << 64) | a[i]) % m;
    return (uint32_t)r;
}

// a * b, schoolbook.
inline Words mul(const Words &a, const Words &b) {
    if (a.empty() || b.empty()) return Words();
    Words r(a.size() + b.size(), 0);
    for (size_t i = 0; i < a.size(); i++) {
        unsigned __int128 carry = 0;
        const uint64_t ai = a[i];
        for (size_t j = 0; j < b.size(); j++) {
            unsigned __int128 t = (unsigned __int128)ai * b[j] + r[i + j] + carry;
            r[i + j] = (uint64_t)t;
            carry = t >> 64;
        }
        r[i + b.size()] = (uint64_t)carry;
    }
    trim(r);
    return r;
}

inline Words mul_small(const Words &a, uint64_t m) {
    Words r(a.size() + 1, 0);
    unsigned __int128 carry = 0;
    for (size_t i = 0; i < a.size(); i++) {
        unsigned __int128 t = (unsigned __int128)a[i] * m + carry;
        r[i] = (uint64_t)t;
        carry = t >> 64;
    }
    r[a.size()] = (uint64_t)carry;
    trim(r);
    return r;
}

inline Words shl(const Words &a, size_t s) {
    if (a.empty()) return a;
    const size_t ws = s / 64, bs = s % 64;
    Words r(a.size() + ws + 1, 0);
    for (size_t i = 0; i < a.size(); i++) {
        r[i + ws] |= a[i] << bs;
        if (bs) r[i + ws + 1] |= a[i] >> (64 - bs);
    }
    trim(r);
    return r;
}

// a - b for a >= b.
inline Words sub(const Words &a, const Words &b) {
    Words r = a;
    uint64_t borrow = 0;
    for (size_t i = 0; i < r.size(); i++) {
        const uint64_t bi = i < b.size() ? b[i] : 0;
        const unsigned __int128 d = (unsigned __int128)r[i] - bi - borrow;
        r[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 127);  // 1 when the subtraction wrapped
    }
    trim(r);
    return r;
}

// r = a * x - b * y for a * x >= b * y (a, b single words); r is reused.
inline void mulsub_small(Words &r, const Words &x, uint64_t a, const Words &y, uint64_t b) {
    const size_t n = std::max(x.size(), y.size()) + 1;
    r.assign(n, 0);
    unsigned __int128 cx = 0, cy = 0;
    uint64_t borrow = 0;
    for (size_t i = 0; i < n; i++) {
        cx += (unsigned __int128)(i < x.size() ? x[i] : 0) * a;
        cy += (unsigned __int128)(i < y.size() ? y[i] : 0) * b;
        const uint64_t px = (uint64_t)cx, py = (uint64_t)cy;
        cx >>= 64;
        cy >>= 64;
        const unsigned __int128 d = (unsigned __int128)px - py - borrow;
        r[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 127);
    }
    trim(r);
}

// r = a * x + b * y (a, b single words); r is reused.
inline void muladd_small(Words &r, const Words &x, uint64_t a, const Words &y, uint64_t b) {
    const size_t n = std::max(x.size(), y.size()) + 2;
    r.assign(n, 0);
    unsigned __int128 cx = 0, cy = 0, c = 0;
    for (size_t i = 0; i < n; i++) {
        cx += (unsigned __int128)(i < x.size() ? x[i] : 0) * a;
        cy += (unsigned __int128)(i < y.size() ? y[i] : 0) * b;
        c += (unsigned __int128)(uint64_t)cx + (uint64_t)cy;
        cx >>= 64;
        cy >>= 64;
        r[i] = (uint64_t)c;
        c >>= 64;
    }
    trim(r);
}

inline Words add(const Words &a, const Words &b) {
    Words r(std::max(a.size(), b.size()) + 1, 0);
    unsigned __int128 c = 0;
    for (size_t i = 0; i < r.size(); i++) {
        c += (unsigned __int128)(i < a.size() ? a[i] : 0) + (i < b.size() ? b[i] : 0);
        r[i] = (uint64_t)c;
        c >>= 64;
    }
    trim(r);
    return r;
}

// Bits sh .. sh + 127 of x.
inline unsigned __int128 bits128(const Words &x, size_t sh) {
    const size_t w = sh / 64, b = sh % 64;
    auto at = [&](size_t i) -> uint64_t { return i < x.size() ? x[i] : 0; };
    const uint64_t w0 = at(w), w1 = at(w + 1), w2 = at(w + 2);
    const uint64_t lo = b ? (w0 >> b) | (w1 << (64 - b)) : w0;
    const uint64_t hi = b ? (w1 >> b) | (w2 << (64 - b)) : w1;
    return ((unsigned __int128)hi << 64) | lo;
}

// a^-1 mod M (0 < a < M) by Lehmer's extended Euclid (Knuth, TAOCP vol. 2,
// 4.5.2, Algorithm L) on 126-bit leading parts, with single-precision
// cofactors kept below 2^62.  Only the cofactor of a is kept, as a
// magnitude and a sign: the remainders u, v satisfy u == tu a, v == tv a
// (mod M), and tu, tv alternate in sign, so every cofactor update adds
// magnitudes.  Returns false when gcd(a, M) != 1.
inline bool inv_mod(const Words &a, const Words &M, Words *inv) {
    Words u = M, v = a, tu, tv(1, 1), u2, v2, t1, t2;
    trim(v);
    int su = -1, sv = 1;  // signs of tu (zero: either) and tv
    const __int128 LIM = (__int128)1 << 62;
    while (!v.empty()) {
        const size_t h = bit_length(u);
        if (h <= 64) {  // single precision to the end
            uint64_t x = u[0], y = v[0];
            while (y) {
                const uint64_t q = x / y, r = x - q * y;
                Words t = add(tu, mul_small(tv, q));  // tu - q tv, magnitude; sign su
                tu = std::move(tv);
                tv = std::move(t);
                std::swap(su, sv);
                x = y;
                y = r;
            }
            u = Words(1, x);
            trim(u);
            v.clear();
            break;
        }
        const size_t sh = h > 126 ? h - 126 : 0;
        __int128 uu = (__int128)bits128(u, sh), vv = (__int128)bits128(v, sh);
        __int128 A = 1, B = 0, C = 0, D = 1;
        while (vv + C != 0 && vv + D != 0) {
            const __int128 q = (uu + A) / (vv + C);
            if (q != (uu + B) / (vv + D)) break;
            const __int128 nC = A - q * C, nD = B - q * D;
            if (nC > LIM || nC < -LIM || nD > LIM || nD < -LIM) break;
            A = C;
            C = nC;
            B = D;
            D = nD;
            const __int128 t = uu - q * vv;
            uu = vv;
            vv = t;
        }
        if (B == 0) {  // no single-precision step was certain: one full division
            Words q, r;
            divmod(u, v, &q, &r);
            Words t = add(tu, mul(tv, q));
            tu = std::move(tv);
            tv = std::move(t);
            std::swap(su, sv);
            u = std::move(v);
            v = std::move(r);
            continue;
        }
        auto mag = [](__int128 x) { return (uint64_t)(x < 0 ? -x : x); };
        // u' = A u + B v, v' = C u + D v (A, B and C, D of opposite signs or
        // zero, u', v' >= 0): the positive term is the one of the
        // non-positive partner's sign opposite (A = 0 after a single step)
        if (B <= 0) mulsub_small(u2, u, mag(A), v, mag(B));
        else mulsub_small(u2, v, mag(B), u, mag(A));
        if (D <= 0) mulsub_small(v2, u, mag(C), v, mag(D));
        else mulsub_small(v2, v, mag(D), u, mag(C));
        // cofactors: A tu and B tv have one sign, as have C tu and D tv
        const int s1 = A != 0 ? (A > 0 ? su : -su) : (B > 0 ? sv : -sv);
        const int s2 = C != 0 ? (C > 0 ? su : -su) : (D > 0 ? sv : -sv);
        muladd_small(t1, tu, mag(A), tv, mag(B));
        muladd_small(t2, tu, mag(C), tv, mag(D));
        std::swap(u, u2);
        std::swap(v, v2);
        std::swap(tu, t1);
        std::swap(tv, t2);
        su = s1;
        sv = s2;
    }
    if (!(u.size() == 1 && u[0] == 1)) return false;
    Words r;
    divmod(tu, M, nullptr, &r);
    if (su < 0 && !r.empty()) r = sub(M, r);
    *inv = r;
    return true;
}

// floor(sqrt(a)) by Newton's iteration from a power of two above the root.
inline Words isqrt(const Words &a) {
    const size_t bits = bit_length(a);
    if (bits == 0) return Words();
    Words x = shl(Words(1, 1), (bits + 1) / 2);
    for (;;) {
        Words q;
        divmod(a, x, &q, nullptr);
        // y = (x + a / x) / 2
        Words y(std::max(x.size(), q.size()) + 1, 0);
        unsigned __int128 c = 0;
        for (size_t i = 0; i < y.size(); i++) {
            c += (unsigned __int128)(i < x.size() ? x[i] : 0) + (i < q.size() ? q[i] : 0);
            y[i] = (uint64_t)c;
            c >>= 64;
        }
        trim(y);
        y = shr(y, 1);
        if (cmp(y, x) >= 0) return x;
        x = y;
    }
}

// 10^e = 5^e * 2^e (square-and-multiply on 5^e).
inline Words pow10(uint64_t e) {
    Words r(1, 1), x(1, 5);
    for (uint64_t k = e; k; k >>= 1) {
        if (k & 1) r = mul(r, x);
        if (k > 1) x = mul(x, x);
    }
    return shl(r, e);
}

}  // namespace big
}  // namespace pfb
