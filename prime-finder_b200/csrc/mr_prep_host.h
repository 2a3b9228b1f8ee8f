// Host set-up of one candidate for the Miller-Rabin engine (the Montgomery
// radix R' = 2^(22 H) + 1 of the transform length, N'' = -N^-1 mod R' by
// Lehmer's extended Euclid, R' mod N, the exponent and its bit cursor; for
// the strong Lucas test Selfridge's parameters and V_0 = 2 in Montgomery
// form): the job GMP does in the reference (barrett.cu:58-107,
// montgomery.cu:30-45).
#pragma once
#include <stdint.h>

#include <vector>

#include "bigint_host.h"
#include "lucas_host.h"
#include "mr_device.cuh"
#include "pfb_mr.h"

namespace pfb {
namespace mr {

struct HostPrep {
    int ok = 0;        // 1 = valid
    int decided = -1;  // >= 0: verdict known without device work (Lucas: a factor, a square)
    int logl = 0;
    int s = 0;
    std::vector<uint32_t> x0, npl, nl, exp;  // R' mod N, N'', N (H limbs each), exponent words
    int cursor = 0;
    int n16 = 0;  // limbs of N (16-bit)
    int q = 0;                 // Lucas: Q
    uint32_t lb = 0;           // Lucas: value bound factor
    std::vector<uint32_t> v0;  // Lucas: V_0 = 2 in Montgomery form
};

inline int choose_logl(size_t nbits, uint32_t base) {
    const int abits = 32 - __builtin_clz(base);
    for (int lg = LOG_LMIN; lg <= LOG_LSEQ; lg++) {
        const size_t rbits = (size_t)LIMB_BITS << (lg - 1);
        if (rbits >= nbits + 2 + 2 * (size_t)abits) return lg;
    }
    return -1;
}

// mode 1: exponent d of N - 1 = 2^s d; mode 0: exponent given; mode 2: the
// strong Lucas test, exponent d of N + 1 = 2^s d.
inline void host_prep(const pfb_mr_number_t &num, uint32_t base, int mode, const pfb_mr_number_t *ex,
                      HostPrep &hp) {
    using namespace pfb::big;
    hp.ok = 0;
    if (!num.limbs || num.n_limbs <= 0) return;
    Words N = from_u16(num.limbs, (size_t)num.n_limbs);
    const size_t nb = bit_length(N);
    if (nb < 2 || !(N[0] & 1ull) || nb > (size_t)PFB_MR_MAX_BITS) return;
    if (mode == 2) {
        long D = 0;
        const int sel = selfridge(N, D);
        if (sel < 0) return;
        if (sel == 0) {
            hp.ok = 1;
            hp.decided = 0;
            return;
        }
        hp.q = (int)((1 - D) / 4);
        const uint32_t aq = (uint32_t)(hp.q < 0 ? -hp.q : hp.q);
        hp.lb = 2u + 4u * aq * aq;
        base = hp.lb;
    }
    int lg = choose_logl(nb, base);
    if (lg < 0) return;
    // N'' = -N^-1 mod R'; when N shares a factor with R' = 2^(22 H) + 1
    // (possible for a prime factor of such a number), the next length's
    // R'' = R'^2 - 2 R' + 2 shares none of them
    Words inv;
    for (; lg <= LOG_LSEQ; lg++) {
        const size_t rb = (size_t)LIMB_BITS << (lg - 1);
        Words M(rb / 64 + 1, 0);
        M[rb / 64] = 1ull << (rb % 64);
        M[0] |= 1ull;
        if (inv_mod(N, M, &inv)) {
            inv = sub(M, inv);
            break;
        }
    }
    if (lg > LOG_LSEQ) return;
    const size_t H = (size_t)1 << (lg - 1);
    const size_t rbits = LIMB_BITS * H;
    Words E;
    int s = 0;
    if (mode == 1) {
        Words nm1 = sub_small(N, 1);
        while (!test_bit(nm1, (size_t)s)) s++;
        E = shr(nm1, (size_t)s);
    } else if (mode == 2) {
        Words np1 = N;
        size_t i = 0;
        while (i < np1.size() && ++np1[i] == 0) i++;
        if (i == np1.size()) np1.push_back(1);
        while (!test_bit(np1, (size_t)s)) s++;
        E = shr(np1, (size_t)s);
    } else {
        if (!ex || !ex->limbs || ex->n_limbs <= 0) return;
        E = from_u16(ex->limbs, (size_t)ex->n_limbs);
        if (E.empty()) return;
    }
    hp.logl = lg;
    hp.s = s;
    hp.n16 = num.n_limbs;
    hp.npl.assign(H, 0);
    hp.nl.assign(H, 0);
    hp.x0.assign(H, 0);
    to_limbs(inv, LIMB_BITS, hp.npl.data(), H);
    to_limbs(N, LIMB_BITS, hp.nl.data(), H);
    Words x0 = add(pow2_mod(rbits, N), Words(1, 1));  // R' mod N
    if (cmp(x0, N) >= 0) x0 = sub(x0, N);
    to_limbs(x0, LIMB_BITS, hp.x0.data(), H);
    if (mode == 2) {
        hp.v0.assign(H, 0);
        to_limbs(mul_small(x0, 2), LIMB_BITS, hp.v0.data(), H);
    }
    const size_t eb = bit_length(E);
    hp.cursor = (int)eb - 1;
    hp.exp.assign((eb + 31) / 32 + 1, 0);
    for (size_t i = 0; i < eb; i++)
        if (test_bit(E, i)) hp.exp[i / 32] |= 1u << (i % 32);
    hp.ok = 1;
}

}  // namespace mr
}  // namespace pfb
