// The reference's C++ Miller-Rabin surface (BatchModCtx, gpu_miller_rabin[_s1],
// miller_rabin.h's miller_rabin_test) implemented on the pfb_mr engine.
#include <stdint.h>
#include <stdio.h>

#include <chrono>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "batch_mod_ctx.cuh"
#include "bigint_host.h"
#include "miller_rabin.h"
#include "miller_rabin_runner.cuh"
#include "pfb_mr.h"

BatchModCtx::BatchModCtx(const std::vector<uint64_t> &N_all, int n_limbs_, int n_batch_, int device_id_)
    : n_limbs(n_limbs_), n_batch(n_batch_), device_id(device_id_) {
    if (n_limbs <= 0 || n_batch <= 0 || N_all.size() < (size_t)n_limbs * (size_t)n_batch)
        throw std::runtime_error("BatchModCtx: N_all holds fewer than n_batch * n_limbs limbs");
    N16.resize((size_t)n_limbs * n_batch);
    for (size_t i = 0; i < N16.size(); i++) {
        if (N_all[i] > 0xFFFFu) throw std::runtime_error("BatchModCtx: limbs must be 16-bit values");
        N16[i] = (uint16_t)N_all[i];
    }
    if (pfb_mr_create(&engine, device_id) != PFB_OK)
        throw std::runtime_error(std::string("BatchModCtx: ") + pfb_last_error());
}

BatchModCtx::~BatchModCtx() { pfb_mr_destroy(engine); }

namespace {

std::vector<bool> run_witnesses(BatchModCtx &mont, int n_total, const std::vector<uint32_t> &witnesses,
                                const char *label, bool show_report) {
    if (n_total < 0 || n_total > mont.n_batch) throw std::runtime_error("gpu_miller_rabin: n_total > n_batch");
    std::vector<bool> alive(n_total, true);
    for (uint32_t w : witnesses) {
        std::vector<int> idx;
        for (int t = 0; t < n_total; t++)
            if (alive[t]) idx.push_back(t);
        if (idx.empty()) break;
        if (show_report) printf("  [%s] witness %-3u alive: %zu\n", label ? label : "", w, idx.size());
        std::vector<pfb_mr_number_t> nums(idx.size());
        for (size_t i = 0; i < idx.size(); i++)
            nums[i] = pfb_mr_number_t{mont.N16.data() + (size_t)idx[i] * mont.n_limbs, mont.n_limbs};
        std::vector<int8_t> ver(idx.size());
        if (pfb_mr_test(mont.engine, nums.data(), (int)nums.size(), w, ver.data(), nullptr, 0) != PFB_OK)
            throw std::runtime_error(std::string("gpu_miller_rabin: ") + pfb_last_error());
        for (size_t i = 0; i < idx.size(); i++)
            if (ver[i] != 1) alive[idx[i]] = false;
    }
    return alive;
}

}  // namespace

std::vector<bool> gpu_miller_rabin_s1(BatchModCtx &mont, const std::vector<uint64_t> &, const std::vector<uint64_t> &,
                                      int n_total, const std::vector<uint32_t> &witnesses, const char *label,
                                      bool show_report, bool) {
    return run_witnesses(mont, n_total, witnesses, label, show_report);
}

std::vector<bool> gpu_miller_rabin(BatchModCtx &mont, const std::vector<uint64_t> &, const std::vector<uint64_t> &,
                                   int, int n_total, const std::vector<uint32_t> &witnesses, const char *label,
                                   bool show_report, bool) {
    return run_witnesses(mont, n_total, witnesses, label, show_report);
}

// ---------------------------------------------------------------------------
// miller_rabin_test: one engine per device, created on first use.

namespace {

std::mutex g_mu;
std::vector<pfb_mr_t *> g_eng;

int ndig(int x) { return x < 10 ? 1 : x < 100 ? 2 : x < 1000 ? 3 : 4; }
int revd(int x, int l) {
    int r = 0;
    for (int i = 0; i < l; i++) {
        r = r * 10 + x % 10;
        x /= 10;
    }
    return r;
}

// 10^a - m1*10^e1 - m2*10^e2 - 1 (miller_rabin.c:56-99); empty on bad input.
pfb::big::Words build(long long a, long long e1, int m1, long long e2, int m2) {
    using namespace pfb::big;
    if (a < 1 || e1 < 0 || e2 < 0 || m1 < 0 || m2 < 0) return Words();
    Words n = pow10((uint64_t)a);
    const Words t1 = mul_small(pow10((uint64_t)e1), (uint64_t)m1);
    const Words t2 = mul_small(pow10((uint64_t)e2), (uint64_t)m2);
    Words one(1, 1);
    Words s = t1;
    {  // s = t1 + t2 + 1
        Words r(std::max(t1.size(), t2.size()) + 1, 0);
        unsigned __int128 carry = 1;
        for (size_t i = 0; i < r.size(); i++) {
            carry += (unsigned __int128)(i < t1.size() ? t1[i] : 0) + (i < t2.size() ? t2[i] : 0);
            r[i] = (uint64_t)carry;
            carry >>= 64;
        }
        trim(r);
        s = r;
    }
    if (cmp(n, s) <= 0) return Words();
    return sub(n, s);
}

// Strong probable-prime rounds to 2, 3, 5, 7, 11 (bases that are multiples of
// a tiny N are skipped); even N and N < 2 are answered directly.
int prp(pfb_mr_t *e, const pfb::big::Words &N) {
    const size_t bits = pfb::big::bit_length(N);
    if (bits <= 1) return 0;                      // 0 or 1
    if (!(N[0] & 1ull)) return bits == 2 ? 1 : 0;  // 2 is prime, other even N are not
    std::vector<uint16_t> l16((bits + 15) / 16);
    pfb::big::to_u16(N, l16.data(), l16.size());
    const pfb_mr_number_t num{l16.data(), (int)l16.size()};
    for (uint32_t base : {2u, 3u, 5u, 7u, 11u}) {
        if (bits <= 4 && base % N[0] == 0) continue;
        int8_t v = -1;
        if (pfb_mr_test(e, &num, 1, base, &v, nullptr, 0) != PFB_OK) return -1;
        if (v != 1) return v < 0 ? -1 : 0;
    }
    return 1;
}

double secs(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

}  // namespace

extern "C" int miller_rabin_test(long long a, long long b, long long c, int k, int j, mr_timing_t *timing) {
    if (timing) *timing = mr_timing_t{0.0, 0.0, 0.0, 0.0};
    if (k < 1 || j < 1 || k > 9999 || j > 9999) return -1;
    pfb_mr_t *e = nullptr;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return -1;
        std::lock_guard<std::mutex> lk(g_mu);
        if ((int)g_eng.size() <= dev) g_eng.resize(dev + 1, nullptr);
        if (!g_eng[dev] && pfb_mr_create(&g_eng[dev], dev) != PFB_OK) return -1;
        e = g_eng[dev];
    }
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    const pfb::big::Words N = build(a, b, k, c, j);
    const auto t1 = clk::now();
    if (N.empty()) return -1;
    const int rN = prp(e, N);
    const auto t2 = clk::now();
    if (timing) {
        timing->build_n = secs(t0, t1);
        timing->mr_n = secs(t1, t2);
    }
    if (rN <= 0) return rN;
    const int lk = ndig(k), lj = ndig(j);
    const pfb::big::Words R = build(a, a - b - lk, revd(k, lk), a - c - lj, revd(j, lj));
    const auto t3 = clk::now();
    if (R.empty()) return -1;
    const int rR = prp(e, R);
    const auto t4 = clk::now();
    if (timing) {
        timing->build_revn = secs(t2, t3);
        timing->mr_revn = secs(t3, t4);
    }
    if (rR < 0) return -1;
    return rR ? 2 : 1;
}
