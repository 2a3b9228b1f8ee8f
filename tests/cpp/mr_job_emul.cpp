// Runs whole tests of the Miller-Rabin engine on the CPU: the engine's own
// host set-up (mr_prep_host.h: host_prep), its set-up kernel and its
// persistent scheduler (mr_kernels.cuh: prep_kernel, persist_kernel ->
// run_job / run_lucas), unchanged, one candidate per CTA, the CTA emulated
// by cooperative fibers (tests/cpp/emul/).  The job state is laid out as
// batch_build (mr.cu) lays it out.
//
// Input lines: "mode base N" (N in hexadecimal; mode 1: strong test to
// `base`, mode 2: strong Lucas test with Selfridge's parameters).  Output
// lines: the verdict (1 probable prime, 0 composite, -1 rejected) and, for
// mode 1, the residue base^d mod N (N - 1 = 2^s d) in hexadecimal.
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "mr_kernels.cuh"
#include "mr_prep_host.h"
#include "mr_tables_host.h"

using namespace pfb::mr;
using pfb::big::Words;

static Words from_hex(const std::string &h) {
    Words w;
    size_t end = h.size();
    while (end > 0) {
        const size_t start = end >= 16 ? end - 16 : 0;
        w.push_back(std::stoull(h.substr(start, end - start), nullptr, 16));
        end = start;
    }
    pfb::big::trim(w);
    return w;
}

static std::string to_hex(Words t) {
    pfb::big::trim(t);
    if (t.empty()) return "0";
    std::string s;
    char buf[24];
    snprintf(buf, sizeof buf, "%llx", (unsigned long long)t.back());
    s += buf;
    for (size_t i = t.size() - 1; i-- > 0;) {
        snprintf(buf, sizeof buf, "%016llx", (unsigned long long)t[i]);
        s += buf;
    }
    return s;
}

int main() {
    const std::vector<uint32_t> h = twiddle_table();
    const int half = 1 << (LOG_LMAX - 1);
    Twiddles tw{};
    for (int pr = 0; pr < 2; pr++) {
        const uint32_t *base = h.data() + (size_t)(4 * pr) * half;
        tw.w[pr] = base;
        tw.wsh[pr] = base + half;
        tw.wi[pr] = base + 2 * half;
        tw.wish[pr] = base + 3 * half;
    }
    c_crt = crt_consts();
    WideTabs wt{};
    const std::vector<uint32_t> wide = wide_tables(h, wt);
    wt.base = reinterpret_cast<const uint4 *>(wide.data());
    c_wide = wt;

    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream in(line);
        int mode = 1;
        uint32_t base = 2;
        std::string sn;
        in >> mode >> base >> sn;
        const Words N = from_hex(sn);
        const size_t n16 = std::max<size_t>(1, (pfb::big::bit_length(N) + 15) / 16);
        std::vector<uint16_t> limbs(n16);
        pfb::big::to_u16(N, limbs.data(), n16);
        const pfb_mr_number_t num{limbs.data(), (int)n16};
        HostPrep hp;
        host_prep(num, base, mode, nullptr, hp);
        if (!hp.ok || hp.decided >= 0) {
            std::cout << (hp.ok ? hp.decided : -1) << (mode == 1 ? " 0" : "") << std::endl;
            continue;
        }
        const int L = 1 << hp.logl, H = L >> 1;
        std::vector<uint32_t> x = hp.x0, res(H), nn(2 * H), nh(2 * H), npl = hp.npl, nl = hp.nl, ex = hp.exp;
        std::vector<uint32_t> yb(H + H / 32);
        std::vector<uint32_t> lv0 = hp.v0, lv1 = hp.x0, lqk = hp.x0, lone = hp.x0, lt(H), gy(2 * L);
        JobDev j{};
        j.x = x.data();
        j.res = res.data();
        j.nn = nn.data();
        j.nh = nh.data();
        j.npl = npl.data();
        j.nl = nl.data();
        j.exp = ex.data();
        if (hp.logl > LOG_LCTA) j.ybuf = yb.data();
        j.logl = hp.logl;
        j.cursor = hp.cursor;
        j.extra = mode >= 1 ? hp.s - 1 : 0;
        j.phase = 0;
        j.base = base;
        j.mode = mode;
        LucasDev lc{};
        if (mode == 2) {
            lv0.resize(H);
            lc.lv0 = lv0.data();
            lc.lv1 = lv1.data();
            lc.lqk = lqk.data();
            lc.lt = lt.data();
            lc.lone = lone.data();
            lc.gy = gy.data();
            lc.q = hp.q;
            lc.lb = hp.lb;
            j.lucas = &lc;
        }
        const size_t smem = smem_bytes(hp.logl);
        emu::run_grid(1, 1, THREADS, [&] { prep_kernel(&j, nullptr, tw); }, smem);
        int locks[1] = {0};
        unsigned counter = 0;
        const int quantum = 64;
        const unsigned total = 4096 / quantum;  // one launch: 4096 steps of the candidate
        for (int launch = 0; j.phase != 3 && launch < 1 << 20; launch++) {
            counter = 0;
            emu::run_grid(1, 1, THREADS, [&] { persist_kernel(&j, 1, locks, &counter, total, quantum, tw); }, smem);
        }
        std::cout << (j.phase == 3 ? j.verdict : -2);
        if (mode == 1) std::cout << " " << to_hex(pfb::big::from_limbs(res.data(), LIMB_BITS, H));
        std::cout << std::endl;
    }
    return 0;
}
