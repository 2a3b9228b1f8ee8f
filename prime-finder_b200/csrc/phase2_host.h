// Host side of Phase 2 shared by miller_rabin_test and the sieve -> test
// pipeline: building N and rev(N) (miller_rabin.c:32-74) and the
// probable-prime decision on the GPU engine.
#pragma once
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "bigint_host.h"
#include "pfb_mr.h"

namespace pfb {
namespace phase2 {

using big::Words;

inline int ndig(int x) { return x < 10 ? 1 : x < 100 ? 2 : x < 1000 ? 3 : 4; }

// Decimal reversal of x written with l digits.
inline int revd(int x, int l) {
    int r = 0;
    for (int i = 0; i < l; i++) {
        r = r * 10 + x % 10;
        x /= 10;
    }
    return r;
}

// P - m1 * Q1 - m2 * Q2 - 1 for non-negative m1, m2; empty if not positive.
inline Words combine(const Words &P, const Words &Q1, uint64_t m1, const Words &Q2, uint64_t m2) {
    using namespace big;
    const Words t1 = mul_small(Q1, m1), t2 = mul_small(Q2, m2);
    Words s(std::max(t1.size(), t2.size()) + 1, 0);
    unsigned __int128 carry = 1;
    for (size_t i = 0; i < s.size(); i++) {
        carry += (unsigned __int128)(i < t1.size() ? t1[i] : 0) + (i < t2.size() ? t2[i] : 0);
        s[i] = (uint64_t)carry;
        carry >>= 64;
    }
    trim(s);
    if (cmp(P, s) <= 0) return Words();
    return sub(P, s);
}

// 10^a - m1*10^e1 - m2*10^e2 - 1 (miller_rabin.c:32-47); empty on a negative
// exponent or a result below 1.
inline Words build(long long a, long long e1, int m1, long long e2, int m2) {
    if (a < 1 || e1 < 0 || e2 < 0 || m1 < 0 || m2 < 0) return Words();
    return combine(big::pow10((uint64_t)a), big::pow10((uint64_t)e1), (uint64_t)m1, big::pow10((uint64_t)e2),
                   (uint64_t)m2);
}

inline Words build_n(long long a, long long b, long long c, int k, int j) { return build(a, b, k, c, j); }

// rev(N) = 10^a - rev(k) 10^(a-b-lk) - rev(j) 10^(a-c-lj) - 1 (miller_rabin.c:56-74).
inline Words build_rev(long long a, long long b, long long c, int k, int j) {
    const int lk = ndig(k), lj = ndig(j);
    return build(a, a - b - lk, revd(k, lk), a - c - lj, revd(j, lj));
}

// Probable-prime decision for many numbers, as GMP's mpz_probab_prime_p(N, 5)
// makes it for the reference (miller_rabin.c:95,107): Baillie-PSW, i.e. the
// strong test to base 2, then the strong Lucas test (Selfridge's parameters)
// on the numbers that pass; each round one batched engine call.  A number
// whose entry in `base2_passed` is non-zero has passed base 2 already.  Even
// numbers and numbers below 2 are answered directly.  Per number: 1 probable
// prime, 0 composite, -1 rejected by the engine (too long).  Returns an empty
// vector if an engine call fails.
inline std::vector<int> prp_batch(pfb_mr_t *e, const std::vector<Words> &nums,
                                  const std::vector<int> *base2_passed = nullptr) {
    const size_t n = nums.size();
    std::vector<int> v(n, 1);
    std::vector<std::vector<uint16_t>> l16(n);
    for (size_t i = 0; i < n; i++) {
        const Words &N = nums[i];
        const size_t bits = big::bit_length(N);
        if (bits <= 1) {
            v[i] = 0;
        } else if (!(N[0] & 1ull)) {
            v[i] = bits == 2 ? 1 : 0;  // 2 is prime, other even N are not
        } else {
            l16[i].resize((bits + 15) / 16);
            big::to_u16(N, l16[i].data(), l16[i].size());
        }
    }
    for (int round = 0; round < 2; round++) {
        std::vector<size_t> idx;
        std::vector<pfb_mr_number_t> q;
        for (size_t i = 0; i < n; i++) {
            if (v[i] != 1 || l16[i].empty()) continue;
            if (round == 0 && base2_passed && (*base2_passed)[i]) continue;
            idx.push_back(i);
            q.push_back(pfb_mr_number_t{l16[i].data(), (int)l16[i].size()});
        }
        if (idx.empty()) continue;
        std::vector<int8_t> ver(idx.size());
        const int rc = round == 0 ? pfb_mr_test(e, q.data(), (int)q.size(), 2u, ver.data(), nullptr, 0)
                                  : pfb_mr_lucas(e, q.data(), (int)q.size(), ver.data());
        if (rc != PFB_OK) return {};
        for (size_t t = 0; t < idx.size(); t++) v[idx[t]] = ver[t] == 1 ? 1 : ver[t] == 0 ? 0 : -1;
    }
    return v;
}

}  // namespace phase2
}  // namespace pfb
