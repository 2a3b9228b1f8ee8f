// Runs the engine's Montgomery step (mr_device.cuh: mont_step, and
// mont_step_seq for L = 2^15) unchanged on the CPU: one CTA of THREADS
// cooperative fibers (tests/cpp/emul/cuda_runtime.h), with the engine's own constant
// tables (mr_tables_host.h) and set-up (bigint_host.h).  Each input line is
//
//   step logl N x a      -> X <- REDC(x^2) * a
//   mul  logl N x y a    -> X <- REDC(x y) * a   (y through its stored spectrum)
//   redc logl N x        -> X <- REDC(x)
//
// with N, x, y in hexadecimal; the output line is X in hexadecimal.  The
// device set-up (NTT of N' and of N, the spectrum of y) follows mr.cu's
// prep_kernel and spectrum for the lengths whose two primes share the CTA,
// and their one-prime-at-a-time form at L = 2^15.
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "bigint_host.h"
#include "mr_device.cuh"
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
                     const CrtConsts &cc, const Spill &sp, const uint32_t *gy) {
    switch (logl) {
        case 8: mont_step<MUL, 8>(sm, cd, square, a, tw, cc, gy); break;
        case 9: mont_step<MUL, 9>(sm, cd, square, a, tw, cc, gy); break;
        case 10: mont_step<MUL, 10>(sm, cd, square, a, tw, cc, gy); break;
        case 14: mont_step<MUL, 14>(sm, cd, square, a, tw, cc, gy); break;
        case 15: mont_step_seq<MUL, 15>(sm, cd, square, a, tw, cc, sp, gy); break;
        default: break;
    }
}

// NTT_n of the zero-padded limbs src (m of them) into g[2][n], both primes, reduced.
static void spectrum(uint32_t *A0, uint32_t *A1, int logn, const uint32_t *src, int m, uint32_t *g,
                     const Twiddles &tw) {
    const int n = 1 << logn, T = (int)blockDim.x, tid = (int)threadIdx.x;
    if (A1) {
        for (int i = tid; i < n; i += T) {
            const uint32_t v = i < m ? src[i] : 0u;
            A0[pad(i)] = v;
            A1[pad(i)] = v;
        }
        __syncthreads();
        dif(A0, A1, logn, tw);
        for (int i = tid; i < n; i += T) {
            g[i] = red2(A0[pad(i)], P1);
            g[n + i] = red2(A1[pad(i)], P2);
        }
        __syncthreads();
        return;
    }
    for (int pr = 0; pr < 2; pr++) {
        for (int i = tid; i < n; i += T) A0[pad(i)] = i < m ? src[i] : 0u;
        __syncthreads();
        if (pr == 0) dif1<0>(A0, logn, tw);
        else dif1<1>(A0, logn, tw);
        const uint32_t p = pr ? P2 : P1;
        for (int i = tid; i < n; i += T) g[pr * n + i] = red2(A0[pad(i)], p);
        __syncthreads();
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
        const bool seq = logl > LOG_LCTA;
        const Words N = from_hex(sn), x = from_hex(sx);
        std::vector<uint32_t> npl(H), nl(H), xl(H), yl(H);
        pfb::big::to_limbs(pfb::big::neg_inv_pow2(N, (size_t)LIMB_BITS * H), LIMB_BITS, npl.data(), H);
        pfb::big::to_limbs(N, LIMB_BITS, nl.data(), H);
        pfb::big::to_limbs(x, LIMB_BITS, xl.data(), H);
        pfb::big::to_limbs(Y, LIMB_BITS, yl.data(), H);
        std::vector<uint32_t> A0(L + L / 32), A1(seq ? 0 : L + L / 32), X(H + H / 32);
        std::vector<uint32_t> nph(2 * L), nh(2 * H), gy(2 * L), ss(L + H + H / 32), st(H);
        CarrySmem cs{};
        uint32_t *a1 = seq ? nullptr : A1.data();
        const Smem sm{A0.data(), a1, X.data(), &cs};
        const Cand cd{nph.data(), nh.data(), logl};
        const Spill sp{ss.data(), st.data()};
        run_cta([&] {
            spectrum(A0.data(), a1, logl, npl.data(), H, nph.data(), tb.tw);
            spectrum(A0.data(), a1, logl - 1, nl.data(), H, nh.data(), tb.tw);
            if (op == "mul") spectrum(A0.data(), a1, logl, yl.data(), H, gy.data(), tb.tw);
            for (int i = (int)threadIdx.x; i < H; i += (int)blockDim.x) X[pad(i)] = xl[i];
            __syncthreads();
            if (op == "mul")
                step_len<true>(logl, sm, cd, false, a, tb.tw, tb.cc, sp, gy.data());
            else
                step_len<false>(logl, sm, cd, op == "step", a, tb.tw, tb.cc, sp, nullptr);
        });
        std::vector<uint32_t> out(H);
        for (int i = 0; i < H; i++) out[i] = X[i + (i >> 5)];
        std::cout << to_hex(pfb::big::from_limbs(out.data(), LIMB_BITS, H)) << std::endl;
    }
    return 0;
}
