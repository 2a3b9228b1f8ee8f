// Line-oriented driver of the host multi-precision helpers (bigint_host.h)
// for the CPU tests: each input line is an operation and hexadecimal
// operands, each output line the hexadecimal result.
//
//   divmod U V        -> quotient remainder
//   pow2_mod e N      -> 2^e mod N              (e decimal)
//   neg_inv N bits    -> -N^-1 mod 2^bits       (bits decimal)
//   inv_mod A M       -> A^-1 mod M, or "-" when gcd(A, M) != 1
//   mul A B / sub A B / shl A s / shr A s / isqrt A / pow10 e / mod_small A m
//   limbs A bits n    -> from_limbs(to_limbs(A)) (round trip through n limbs)
//   u16 A n           -> from_u16(to_u16(A))     (round trip through n limbs)
//   build a b c k j r -> N (r = 0) or rev(N) (r = 1) of phase2_host.h, "-" if
//                        the reference formula gives no positive number
//   selfridge N       -> "1 D" (Selfridge's D), "0" (composite found), "-1"
#include <cstdio>
#include <iostream>
#include <sstream>
#include <string>

#include "bigint_host.h"
#include "lucas_host.h"
#include "phase2_host.h"

using namespace pfb::big;

static Words from_hex(const std::string &h) {
    Words w;
    size_t end = h.size();
    while (end > 0) {
        const size_t start = end >= 16 ? end - 16 : 0;
        w.push_back(std::stoull(h.substr(start, end - start), nullptr, 16));
        end = start;
    }
    trim(w);
    return w;
}

static std::string to_hex(const Words &a) {
    Words t = a;
    trim(t);
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
    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream in(line);
        std::string op, x, y, z;
        in >> op >> x >> y >> z;
        if (op == "divmod") {
            Words q, r;
            divmod(from_hex(x), from_hex(y), &q, &r);
            std::cout << to_hex(q) << " " << to_hex(r) << "\n";
        } else if (op == "pow2_mod") {
            std::cout << to_hex(pow2_mod(std::stoull(x), from_hex(y))) << "\n";
        } else if (op == "neg_inv") {
            std::cout << to_hex(neg_inv_pow2(from_hex(x), std::stoull(y))) << "\n";
        } else if (op == "inv_mod") {
            Words r;
            std::cout << (inv_mod(from_hex(x), from_hex(y), &r) ? to_hex(r) : std::string("-")) << "\n";
        } else if (op == "mul") {
            std::cout << to_hex(mul(from_hex(x), from_hex(y))) << "\n";
        } else if (op == "sub") {
            std::cout << to_hex(sub(from_hex(x), from_hex(y))) << "\n";
        } else if (op == "shl") {
            std::cout << to_hex(shl(from_hex(x), std::stoull(y))) << "\n";
        } else if (op == "shr") {
            std::cout << to_hex(shr(from_hex(x), std::stoull(y))) << "\n";
        } else if (op == "isqrt") {
            std::cout << to_hex(isqrt(from_hex(x))) << "\n";
        } else if (op == "pow10") {
            std::cout << to_hex(pow10(std::stoull(x))) << "\n";
        } else if (op == "mod_small") {
            std::cout << mod_small(from_hex(x), (uint32_t)std::stoul(y)) << "\n";
        } else if (op == "limbs") {
            const unsigned bits = (unsigned)std::stoul(y);
            const size_t n = std::stoull(z);
            std::vector<uint32_t> l(n);
            to_limbs(from_hex(x), bits, l.data(), n);
            std::cout << to_hex(from_limbs(l.data(), bits, n)) << "\n";
        } else if (op == "u16") {
            const size_t n = std::stoull(y);
            std::vector<uint16_t> l(n);
            to_u16(from_hex(x), l.data(), n);
            std::cout << to_hex(from_u16(l.data(), n)) << "\n";
        } else if (op == "build") {
            long long v[6] = {0, 0, 0, 0, 0, 0};
            std::istringstream all(line.substr(op.size()));
            for (auto &t : v) all >> t;
            const Words w = v[5] ? pfb::phase2::build_rev(v[0], v[1], v[2], (int)v[3], (int)v[4])
                                 : pfb::phase2::build_n(v[0], v[1], v[2], (int)v[3], (int)v[4]);
            std::cout << (w.empty() ? std::string("-") : to_hex(w)) << "\n";
        } else if (op == "selfridge") {
            long D = 0;
            const int r = pfb::mr::selfridge(from_hex(x), D);
            if (r == 1) std::cout << "1 " << D << "\n";
            else std::cout << r << "\n";
        } else {
            std::cout << "?\n";
        }
    }
    return 0;
}
