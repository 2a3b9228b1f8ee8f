// Runs the engine's Montgomery step (mr_device.cuh: mont_step, the radix
// R' = 2^(22 H) + 1) unchanged on the CPU: one CTA of THREADS cooperative
// fibers (tests/cpp/emul/cuda_runtime.h), with the engine's own constant
// tables (mr_tables_host.h), set-up of N'' (bigint_host.h: inv_mod) and
// spectra (mr_kernels.cuh: spectra_t, spectrum).  Each input line is
//
//   step logl N x a      -> X <- REDC(x^2) * a
//   mul  logl N x y a    -> X <- REDC(x y) * a   (y through its stored spectrum)
//   redc logl N x        -> X <- REDC(x)
//
// with N, x, y in hexadecimal; the output line is X in hexadecimal.  Every
// buffer is a host array of exactly the size the kernel's layout gives it.
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "bigint_host.h"
#include "mr_kernels.cuh"
#include "mr_tables_host.h"

using namespace pfb::mr;
using pfb::big::Words;

static void run_cta(const std::function<void()> &f) { emu::run_cta(THREADS, f); }

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

struct Tables {
    std::vector<uint32_t> h, wide;
    Twiddles tw{};
    CrtConsts cc{};
    Tables() {
        h = twiddle_table();
        const int half = 1 << (LOG_LMAX - 1);
        for (int pr = 0; pr < 2; pr++) {
            const uint32_t *base = h.data() + (size_t)(4 * pr) * half;
            tw.w[pr] = base;
            tw.wsh[pr] = base + half;
            tw.wi[pr] = base + 2 * half;
            tw.wish[pr] = base + 3 * half;
        }
        cc = crt_consts();
        WideTabs wt{};
        wide = wide_tables(h, wt);
        wt.base = reinterpret_cast<const uint4 *>(wide.data());
        c_wide = wt;
    }
};

template <bool MUL>
static void step_len(int logl, const Smem &sm, const Cand &cd, bool square, uint32_t a, const Twiddles &tw,
                     const CrtConsts &cc, const uint32_t *gy) {
    switch (logl) {
        case 8: mont_step<MUL, 8>(sm, cd, square, a, tw, cc, gy); break;
        case 9: mont_step<MUL, 9>(sm, cd, square, a, tw, cc, gy); break;
        case 10: mont_step<MUL, 10>(sm, cd, square, a, tw, cc, gy); break;
        case 14: mont_step<MUL, 14>(sm, cd, square, a, tw, cc, gy); break;
        case 15: mont_step<MUL, 15>(sm, cd, square, a, tw, cc, gy); break;
        default: break;
    }
}

int main() {
    const Tables tb;
    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream in(line);
        std::string op, sl, sn, sx, sy;
        in >> op >> sl >> sn >> sx;
        const int logl = std::stoi(sl);
        uint32_t a = 1;
        Words Y;
        if (op == "mul") {
            in >> sy >> a;
            Y = from_hex(sy);
        } else if (op == "step") {
            in >> a;
        }
        const int L = 1 << logl, H = L >> 1;
        const Words N = from_hex(sn), x = from_hex(sx);
        // N'' = -N^-1 mod (2^(22 H) + 1)
        const size_t rb = (size_t)LIMB_BITS * H;
        Words M(rb / 64 + 1, 0), inv;
        M[rb / 64] = 1ull << (rb % 64);
        M[0] |= 1ull;
        if (!pfb::big::inv_mod(N, M, &inv)) {
            std::cout << "-" << std::endl;
            continue;
        }
        inv = pfb::big::sub(M, inv);
        std::vector<uint32_t> npl(H), nl(H), xl(H), yl(H);
        pfb::big::to_limbs(inv, LIMB_BITS, npl.data(), H);
        pfb::big::to_limbs(N, LIMB_BITS, nl.data(), H);
        pfb::big::to_limbs(x, LIMB_BITS, xl.data(), H);
        pfb::big::to_limbs(Y, LIMB_BITS, yl.data(), H);
        const int B = H + H / 32, BA = logl <= LOG_LCTA ? L + L / 32 : B;
        std::vector<uint32_t> A0(BA), A1(BA), X(B);
        std::vector<uint32_t> nn(2 * H), nh(2 * H), gy(2 * L);
        CarrySmem cs{};
        const Smem sm{A0.data(), A1.data(), X.data(), &cs};
        const Cand cd{nn.data(), nh.data(), logl};
        run_cta([&] {
            switch (logl) {
                case 8: spectra_t<8>(sm, npl.data(), nullptr, nullptr, nn.data(), nn.data() + H, tb.tw, false); break;
                case 9: spectra_t<9>(sm, npl.data(), nullptr, nullptr, nn.data(), nn.data() + H, tb.tw, false); break;
                case 10: spectra_t<10>(sm, npl.data(), nullptr, nullptr, nn.data(), nn.data() + H, tb.tw, false); break;
                case 14: spectra_t<14>(sm, npl.data(), nullptr, nullptr, nn.data(), nn.data() + H, tb.tw, false); break;
                case 15: spectra_t<15>(sm, npl.data(), nullptr, nullptr, nn.data(), nn.data() + H, tb.tw, false); break;
            }
            spectrum(sm, logl, nl.data(), gy.data(), tb.tw);  // cyclic half of N: gy[0..H), gy[L..L+H)
            for (int i = (int)threadIdx.x; i < H; i += (int)blockDim.x) {
                nh[i] = gy[i];
                nh[H + i] = gy[L + i];
            }
            __syncthreads();
            if (op == "mul") spectrum(sm, logl, yl.data(), gy.data(), tb.tw);
            for (int i = (int)threadIdx.x; i < H; i += (int)blockDim.x) X[pad(i)] = xl[i];
            __syncthreads();
            if (op == "mul")
                step_len<true>(logl, sm, cd, false, a, tb.tw, tb.cc, gy.data());
            else
                step_len<false>(logl, sm, cd, op == "step", a, tb.tw, tb.cc, nullptr);
        });
        std::vector<uint32_t> out(H);
        for (int i = 0; i < H; i++) out[i] = X[i + (i >> 5)];
        std::cout << to_hex(pfb::big::from_limbs(out.data(), LIMB_BITS, H)) << std::endl;
    }
    return 0;
}
