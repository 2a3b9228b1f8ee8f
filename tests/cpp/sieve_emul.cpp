// Runs the Phase-1 sieve kernels (sieve_device.cuh) unchanged on the CPU, one
// CTA after another, each CTA as cooperative fibers (tests/cpp/emul/).  The
// launches are those pfb_sieve_run and pfb_sieve_survivors make for one
// triple (sieve.cu: ensure_split, enqueue_sieve, pfb_sieve_survivors).
//
// Input: "K a b c [compact [unique]]", then "n p_1 ... p_n" (the prime list).
// unique = 1 splits the list as pfb_sieve_run_noalloc does (split_unique_kernel:
// repeated entries listed once, into lists of fixed capacity).
// Output: the mask as hexadecimal little-endian words (one line), then the
// number of survivors and the 64-bit FNV-1a hash of the survivor list
// (k<<16|j as little-endian uint32), in decimal (one line; "0 0" when
// compact is given as 0 and the compaction is skipped).
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

#include "sieve_device.cuh"

int main() {
    int K = 0;
    long long abc[3] = {0, 0, 0};
    uint32_t n = 0;
    std::string first;
    std::getline(std::cin, first);
    std::istringstream f(first);
    int compact = 1, unique = 0;
    f >> K >> abc[0] >> abc[1] >> abc[2];
    if (!(f >> compact)) compact = 1;
    if (!(f >> unique)) unique = 0;
    std::cin >> n;
    std::vector<uint32_t> primes(n ? n : 1);
    for (uint32_t i = 0; i < n; i++) std::cin >> primes[i];
    if (!std::cin || K < 1 || K > PFB_SIEVE_MAX_K) return 2;

    const size_t wpt = ((size_t)K * (size_t)K + 31u) / 32u;  // words of pfb_sieve_mask_bytes(K)
    std::vector<uint32_t> mask(wpt, 0u);
    // split of the prime list (ensure_split): a grid-stride kernel, any grid
    const uint32_t lim = small_limit(K), cap = lim / 2u + 2u;
    std::vector<uint32_t> tiny(cap), small(cap), counts(2, 0u);
    std::vector<uint32_t> seen(lim / 32u + 1u, 0u);
    if (n && unique)
        emu::run_grid(4, 1, 256, [&] {
            split_unique_kernel(primes.data(), n, lim, seen.data(), tiny.data(), small.data(), counts.data());
        });
    else if (n)
        emu::run_grid(4, 1, 256, [&] { split_kernel(primes.data(), n, lim, cap, tiny.data(), small.data(), counts.data()); });
    if (counts[0] > cap || counts[1] > cap) return 3;
    const uint32_t n_small_all = counts[0] + counts[1];
    // small primes (enqueue_sieve): line records, then row tiles in shared memory
    std::vector<SmallRec> rec(2 * cap);
    if (n_small_all) {
        emu::run_grid((n_small_all + 127u) / 128u, 1, 128, [&] {
            small_setup_kernel(tiny.data(), small.data(), counts.data(), abc, 1, K, 2u * cap, rec.data());
        });
        const uint32_t tiles = ((uint32_t)K + kTileRows - 1u) / kTileRows;
        const uint32_t rows = (uint32_t)K < (uint32_t)kTileRows ? (uint32_t)K : (uint32_t)kTileRows;
        emu::run_grid(tiles, 1, kBlockTile, [&] {
            small_tile_kernel(rec.data(), counts.data(), 2u * cap, abc, K, mask.data(), wpt);
        }, tile_smem_bytes(rows, K));
    }
    // medium primes (a warp per prime, a small grid so that the warps take
    // several batches) and large primes (one thread per prime of the list)
    const uint32_t p_med = medium_limit(K, lim);
    if (n) {
        auto large = [&](auto dc) {
            constexpr int D = decltype(dc)::value;
            if (p_med > lim)
                emu::run_grid(2, 1, kBlockLarge, [&] {
                    medium_kernel<D>(primes.data(), n, lim, p_med, abc, K, mask.data(), wpt);
                });
            emu::run_grid((n + kBlockLarge - 1) / kBlockLarge, 1, kBlockLarge, [&] {
                large_kernel<D>(primes.data(), n, p_med, abc, K, mask.data(), wpt);
            });
        };
        switch (ndigits(K)) {
        case 1: large(std::integral_constant<int, 1>()); break;
        case 2: large(std::integral_constant<int, 2>()); break;
        case 3: large(std::integral_constant<int, 3>()); break;
        default: large(std::integral_constant<int, 4>()); break;
        }
    }
    // survivor compaction (pfb_sieve_survivors)
    const uint32_t nbits = (uint32_t)K * (uint32_t)K, nwords = (nbits + 31u) / 32u, chunks = (nwords + 31u) / 32u;
    std::vector<uint32_t> chunk(chunks), out(compact ? nbits : 1);
    uint32_t total = 0;
    if (compact) {
        emu::run_grid(chunks, 1, 32, [&] { surv_count_kernel(mask.data(), nbits, chunk.data()); });
        emu::run_grid(1, 1, 1024, [&] { surv_scan_kernel(chunk.data(), chunks, &total); });
        emu::run_grid(chunks, 1, 32, [&] {
            surv_write_kernel(mask.data(), nbits, K, chunk.data(), out.data(), nbits);
        });
    }
    char buf[16];
    for (size_t i = 0; i < wpt; i++) {
        snprintf(buf, sizeof buf, "%08x", mask[i]);
        std::cout << buf;
    }
    unsigned long long h = 1469598103934665603ull;  // FNV-1a 64
    for (uint32_t i = 0; i < total && i < nbits; i++)
        for (int byte = 0; byte < 4; byte++) {
            h ^= (out[i] >> (8 * byte)) & 0xFFu;
            h *= 1099511628211ull;
        }
    std::cout << "\n" << total << " " << h << "\n";
    return 0;
}
