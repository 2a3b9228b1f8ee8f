// Runs the per-operation modular context (mr_ctx_kernels.cuh: ctx_kernel, the
// device side of pfb_mr_ctx_* / BatchModCtx) on the CPU: the engine's own
// host set-up (host_prep), set-up kernel (prep_kernel) and ctx_kernel,
// unchanged, one modulus per CTA, the CTA emulated by cooperative fibers
// (tests/cpp/emul/), with the modulus' buffers laid out as pfb_mr_ctx_create
// lays them out.
//
// Input lines: "op n16 N A [B]" (op: 0 modsq, 1 modmul, 2 raw square, 3 raw
// product, 4 from working form; N, A, B in hexadecimal; n16 = 16-bit limbs
// per operand).  Output lines: "logl result" (result in hexadecimal), or
// "-1" for a modulus the set-up rejects.
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "mr_ctx_kernels.cuh"
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

static std::vector<uint64_t> limbs64(const Words &w, int n16) {
    std::vector<uint16_t> t(n16);
    pfb::big::to_u16(w, t.data(), (size_t)n16);
    return std::vector<uint64_t>(t.begin(), t.end());
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
        int op = 0, n16 = 0;
        std::string sn, sa, sb;
        in >> op >> n16 >> sn >> sa;
        if (!(in >> sb)) sb = "0";
        const Words N = from_hex(sn);
        const std::vector<uint64_t> nall = limbs64(N, n16);
        std::vector<uint16_t> n16v(nall.begin(), nall.end());
        const pfb_mr_number_t num{n16v.data(), n16};
        HostPrep hp;
        host_prep(num, 2u, 1, nullptr, hp);
        if (!hp.ok) {
            std::cout << -1 << std::endl;
            continue;
        }
        const int L = 1 << hp.logl, H = L >> 1;
        std::vector<uint32_t> x(H), res(H), nn(2 * H), nh(2 * H), npl = hp.npl, nl = hp.nl;
        std::vector<uint32_t> yb(H + H / 32), gy(2 * L), yl(H);
        std::vector<unsigned long long> rawc(L);
        JobDev j{};
        j.x = x.data();
        j.res = res.data();
        j.nn = nn.data();
        j.nh = nh.data();
        j.npl = npl.data();
        j.nl = nl.data();
        if (hp.logl > LOG_LCTA) j.ybuf = yb.data();
        j.logl = hp.logl;
        j.phase = 0;
        CtxExtra ex{gy.data(), yl.data(), rawc.data()};
        const size_t smem = smem_bytes(hp.logl);
        emu::run_grid(1, 1, THREADS, [&] { prep_kernel(&j, nullptr, tw); }, smem);
        const std::vector<uint64_t> A = limbs64(from_hex(sa), n16), B = limbs64(from_hex(sb), n16);
        const int n_sum = 2 * n16 + 16;
        const int out_stride = (op == CTX_RAW_SQ || op == CTX_RAW_MUL) ? n_sum : n16;
        std::vector<uint64_t> out(out_stride, 0xDEADu);
        emu::run_grid(1, 1, THREADS, [&] {
            ctx_kernel(&j, &ex, A.data(), B.data(), out.data(), n16, out_stride, op, tw);
        }, smem);
        std::vector<uint16_t> o16(out.begin(), out.end());
        for (uint64_t v : out)
            if (v > 0xFFFFu) o16[0] = 0, std::cerr << "limb above 16 bits\n";
        std::cout << hp.logl << " " << to_hex(pfb::big::from_u16(o16.data(), o16.size())) << std::endl;
    }
    return 0;
}
