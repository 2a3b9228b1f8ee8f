// The engine's carry machinery (mr_device.cuh: carry_pass, end_around) run
// unchanged on the CPU, one CTA of THREADS cooperative fibers, against
// 128-bit host arithmetic.
//
//   carry_pass: n raw coefficients below 2^62 (random, all B - 1, or zero
//   runs) and a carry-in; the limbs and the carry out must equal a serial
//   carry over the whole array.
//   end_around: X + c mod B^H - 1 for X with limbs 2..k all B - 1 (k up to
//   H - 1, so the warp ripple and the fallback passes both run) and random c
//   below 2^44; compared with a serial end-around addition.
//
// Prints "ok <cases>" or the first mismatch.
#include <cstdio>
#include <functional>
#include <random>
#include <vector>

#include "mr_device.cuh"

using namespace pfb::mr;

int main() {
    std::mt19937_64 rng(7);
    long long cases = 0;
    for (int logn = 7; logn <= 15; logn++) {
        const int n = 1 << logn;
        for (int it = 0; it < 6; it++) {
            std::vector<unsigned long long> raw(n);
            for (int i = 0; i < n; i++) {
                switch (it % 3) {
                case 0: raw[i] = rng() >> 2; break;
                case 1: raw[i] = LIMB_MASK; break;
                default: raw[i] = (i % 97 < 50) ? LIMB_MASK : (rng() >> 30); break;
                }
            }
            const unsigned long long cin = it < 3 ? (rng() >> 23) : 1ull;
            std::vector<uint32_t> out(n + n / 32 + 1, 0u), want(n);
            unsigned __int128 acc = cin;
            for (int i = 0; i < n; i++) {
                acc += raw[i];
                want[i] = (uint32_t)(acc & LIMB_MASK);
                acc >>= LIMB_BITS;
            }
            CarrySmem cs{};
            unsigned long long got = 0;
            emu::run_cta(THREADS, [&] {
                const unsigned long long r = carry_pass<true>(n, cin, [&](int i) { return raw[i]; }, out.data(), cs);
                if (threadIdx.x == 0) got = r;
            });
            for (int i = 0; i < n; i++)
                if (out[pad(i)] != want[i]) {
                    printf("carry_pass limb mismatch n=%d it=%d i=%d\n", n, it, i);
                    return 1;
                }
            if (got != (unsigned long long)acc) {
                printf("carry_pass carry mismatch n=%d it=%d\n", n, it);
                return 1;
            }
            cases++;
        }
    }
    for (int logh = 7; logh <= 14; logh++) {
        const int H = 1 << logh;
        for (int k : {1, 2, 5, 31, 32, 33, 100, H - 2, H - 1}) {
            if (k >= H) continue;
            for (int it = 0; it < 4; it++) {
                std::vector<uint32_t> lim(H);
                for (int i = 0; i < H; i++) lim[i] = (uint32_t)(rng() & LIMB_MASK);
                for (int i = 2; i <= k; i++) lim[i] = LIMB_MASK;
                if (it == 3) lim[0] = lim[1] = LIMB_MASK;
                const unsigned long long c = (rng() >> 20) | 1ull;  // below 2^44, not 0
                // serial: X + c, end-around carries until none is left
                std::vector<uint32_t> want = lim;
                unsigned long long carry = c;
                while (carry) {
                    unsigned __int128 a = carry;
                    for (int i = 0; i < H; i++) {
                        a += want[i];
                        want[i] = (uint32_t)(a & LIMB_MASK);
                        a >>= LIMB_BITS;
                    }
                    carry = (unsigned long long)a;
                }
                std::vector<uint32_t> X(H + H / 32 + 1, 0u);
                for (int i = 0; i < H; i++) X[pad(i)] = lim[i];
                CarrySmem cs{};
                emu::run_cta(THREADS, [&] { end_around(X.data(), c, H, cs); });
                for (int i = 0; i < H; i++)
                    if (X[pad(i)] != want[i]) {
                        printf("end_around mismatch H=%d k=%d it=%d i=%d\n", H, k, it, i);
                        return 1;
                    }
                cases++;
            }
        }
    }
    printf("ok %lld\n", cases);
    return 0;
}
