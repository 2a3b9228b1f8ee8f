// Caller of the C++ / C drop-in surface, compiled against include/ and
// libpfb200.so by tests/test_cpp_api_gpu.py.  Prints one line per check.
//   mersenne <p> <alive>           BatchModCtx + gpu_miller_rabin_s1, 16 witnesses
//   mrt <a> <b> <c> <k> <j> <ret>  miller_rabin_test
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "miller_rabin.h"
#include "miller_rabin_runner.cuh"

int main(int argc, char **argv) {
    const int ps[] = {521, 607, 1279};
    const int n_limbs = 1279 / 16 + 2;
    std::vector<uint64_t> N_all(3 * (size_t)n_limbs, 0), dummy;
    for (int i = 0; i < 3; i++)
        for (int bit = 0; bit < ps[i]; bit++) N_all[(size_t)i * n_limbs + bit / 16] |= 1ull << (bit % 16);
    BatchModCtx mont(N_all, n_limbs, 3);
    std::vector<bool> alive = gpu_miller_rabin_s1(mont, dummy, dummy, 3, DEFAULT_WITNESSES, "Mersenne");
    for (int i = 0; i < 3; i++) printf("mersenne %d %d\n", ps[i], (int)alive[i]);
    for (int i = 1; i + 4 < argc; i += 5) {
        const long long a = atoll(argv[i]), b = atoll(argv[i + 1]), c = atoll(argv[i + 2]);
        const int k = atoi(argv[i + 3]), j = atoi(argv[i + 4]);
        mr_timing_t t;
        printf("mrt %lld %lld %lld %d %d %d\n", a, b, c, k, j, miller_rabin_test(a, b, c, k, j, &t));
    }
    return 0;
}
