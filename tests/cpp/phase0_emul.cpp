// Runs the Phase-0 kernels (phase0_device.cuh) unchanged on the CPU, CTA
// after CTA, each CTA as cooperative fibers (tests/cpp/emul/): the table
// entries as pfb_phase0_create builds them, build_kernel over every mask of
// the table (grid-stride, a small grid), then apply_kernel as
// pfb_phase0_apply launches it (one CTA per triple).
//
// Input: "n p_1 ... p_n" (the small primes), then "m a_1 b_1 c_1 ... a_m b_m
// c_m".  Output: one line per triple, its 313 mask words in hexadecimal.
#include <functional>
#include <iostream>
#include <vector>

#include "phase0_device.cuh"

int main() {
    uint32_t n = 0;
    std::cin >> n;
    std::vector<uint32_t> primes(n ? n : 1);
    for (uint32_t i = 0; i < n; i++) std::cin >> primes[i];
    int m = 0;
    std::cin >> m;
    std::vector<long long> abc(3 * (size_t)(m > 0 ? m : 1));
    for (int i = 0; i < 3 * m; i++) std::cin >> abc[i];
    if (!std::cin || m <= 0) return 2;

    std::vector<Entry> ent;
    std::vector<uint32_t> pw, ipw;
    long long cells = 0, words = 0;
    phase0_tables(primes.data(), n, ent, pw, ipw, cells, words);
    std::vector<uint32_t> table((size_t)words);
    std::vector<uint32_t> masks((size_t)m * kWords, 0u);
    const int n_ent = (int)ent.size();
    if (n_ent > 0) {
        emu::run_grid(8, 1, kBuildThreads, [&] {
            build_kernel(ent.data(), n_ent, pw.data(), ipw.data(), cells, table.data());
        });
        emu::run_grid((unsigned)m, 1, kApplyThreads, [&] {
            apply_kernel(ent.data(), n_ent, table.data(), abc.data(), masks.data(), 0);
        });
    }
    char buf[16];
    for (int t = 0; t < m; t++) {
        for (int w = 0; w < kWords; w++) {
            snprintf(buf, sizeof buf, "%08x", masks[(size_t)t * kWords + w]);
            std::cout << buf;
        }
        std::cout << "\n";
    }
    return 0;
}
