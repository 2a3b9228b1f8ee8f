"""The engine's host multi-precision helpers (prime-finder_b200/csrc/bigint_host.h)
against Python integers, on the CPU.

These compute the per-modulus set-up the reference does with GMP
(barrett.cu:58-107, montgomery.cu:30-45): N' = -N^-1 mod 2^bits by Hensel
lifting, 2^e mod N by Knuth's long division, the candidate's powers of ten,
the limb conversions between the reference's 16-bit format and the
engine's 22-bit limbs, and the candidates N and rev(N) that miller_rabin_test
and the sieve -> test pipeline build (phase2_host.h, miller_rabin.c:32-74),
against the oracle's restatement of the reference's build_N/build_revN, and
Selfridge's parameters for the strong Lucas test (lucas_host.h) against the
oracle's restatement (oracle/lucas.py).  A small driver (tests/cpp/bigint_host_check.cpp)
is compiled against the header and fed random and edge-case operands.
"""
import math
import os
import random
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.set_int_max_str_digits(0)


@pytest.fixture(scope="module")
def run(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("bigint") / "bigint_host_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "prime-finder_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "bigint_host_check.cpp"), "-o", exe], check=True)

    def go(lines):
        out = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True,
                             check=True).stdout.split("\n")
        return out[:len(lines)]
    return go


def h(x):
    return format(x, "x")


def _candidate(a, b, c, k, j):
    return 10 ** a - k * 10 ** b - j * 10 ** c - 1


def test_divmod(run):
    rng = random.Random(1)
    cases = []
    for _ in range(150):
        nb = rng.choice([32, 64, 65, 200, 1000, 5000])
        v = rng.getrandbits(nb) | 1
        u = rng.getrandbits(nb + rng.choice([0, 1, 31, 32, 33, 300, 3000]))
        cases.append((u, v))
    cases += [(0, 5), (7, 7), (6, 7), (14, 7), ((1 << 640) - 1, (1 << 320) - 1), (1 << 500, (1 << 64) + 1)]
    # a quotient digit estimate that is one too large (the add-back step of algorithm D)
    cases.append(((0x7FFFFFFF << 96) | (0x80000000 << 64), (0x80000000 << 64) | 1))
    cases.append(((0x7FFF800000000000 << 128), (0x800000000000 << 64) + 1))
    N = _candidate(3000, 1700, 100, 7, 19)
    cases.append((N * N + 12345, N))
    out = run(["divmod %s %s" % (h(u), h(v)) for u, v in cases])
    for (u, v), line in zip(cases, out):
        q, r = (int(t, 16) for t in line.split())
        assert (q, r) == divmod(u, v), (u, v)


def test_pow2_mod_and_neg_inv_at_transform_sizes(run):
    """The set-up of a 50 000-digit candidate at L = 2^14 (R = 2^(22 * 8192))
    and of smaller ones at other lengths."""
    rng = random.Random(2)
    Ns = [_candidate(50000, 30000, 100, 1, 99), _candidate(2000, 1000, 100, 5, 84)]
    Ns += [rng.getrandbits(b) | 1 | (1 << (b - 1)) for b in (3, 63, 64, 65, 700, 4000)]
    lines, want = [], []
    for N in Ns:
        rbits = 22 * 8192 if N.bit_length() > 100000 else 22 * (1 << max(1, (N.bit_length() // 22 + 2).bit_length()))
        lines.append("pow2_mod %d %s" % (rbits, h(N)))
        want.append(pow(2, rbits, N))
        lines.append("neg_inv %s %d" % (h(N), rbits))
        want.append((-pow(N, -1, 1 << rbits)) % (1 << rbits))
    out = run(lines)
    assert [int(x, 16) for x in out] == want


def test_arithmetic_and_shifts(run):
    rng = random.Random(3)
    lines, want = [], []
    for _ in range(60):
        a = rng.getrandbits(rng.choice([1, 64, 65, 128, 900]))
        b = rng.getrandbits(rng.choice([1, 64, 65, 128, 900]))
        s = rng.choice([0, 1, 63, 64, 65, 200])
        lines += ["mul %s %s" % (h(a), h(b)), "sub %s %s" % (h(max(a, b)), h(min(a, b))),
                  "shl %s %d" % (h(a), s), "shr %s %d" % (h(a), s)]
        want += [a * b, max(a, b) - min(a, b), a << s, a >> s]
    for m in (3, 7, 65521, 4294967291):
        a = rng.getrandbits(3000)
        lines.append("mod_small %s %d" % (h(a), m))
        want.append(a % m)
    out = run(lines)
    got = [int(x, 16) if not l.startswith("mod_small") else int(x) for l, x in zip(lines, out)]
    assert got == want


def test_isqrt(run):
    rng = random.Random(4)
    vals = [1, 2, 3, 4, 15, 16, 17, (1 << 128) - 1, 1 << 128]
    for b in (40, 200, 2000):
        r = rng.getrandbits(b)
        vals += [r * r - 1, r * r, r * r + 1, r * r + 2 * r]
    out = run(["isqrt %s" % h(v) for v in vals])
    assert [int(x, 16) for x in out] == [math.isqrt(v) for v in vals]


def test_pow10(run):
    es = [0, 1, 2, 19, 20, 27, 28, 100, 1001, 50000]
    out = run(["pow10 %d" % e for e in es])
    assert [int(x, 16) for x in out] == [10 ** e for e in es]


def test_limb_round_trips(run):
    rng = random.Random(5)
    lines, want = [], []
    for bits in (16, 22, 32):
        for n in (1, 2, 3, 7, 8192):
            a = rng.getrandbits(bits * n)
            lines.append("limbs %s %d %d" % (h(a), bits, n))
            want.append(a)
            # truncation: only the low n limbs are kept
            big = a | (rng.getrandbits(50) << (bits * n))
            lines.append("limbs %s %d %d" % (h(big), bits, n))
            want.append(a)
    for n in (1, 4, 5, 10386):
        a = rng.getrandbits(16 * n)
        lines.append("u16 %s %d" % (h(a), n))
        want.append(a)
    out = run(lines)
    assert [int(x, 16) for x in out] == want


def test_candidates_equal_the_reference_formula(run):
    """N = 10^a - k 10^b - j 10^c - 1 and rev(N) = 10^a - rev(k) 10^(a-b-lk)
    - rev(j) 10^(a-c-lj) - 1, including the tuples where rev(N) is not the
    literal digit reversal (overlapping blocks, b + lk >= a) and the ones with
    a negative exponent or a non-positive result, which both reject."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    rng = random.Random(6)
    tuples = [(50000, 30000, 100, 1, 99), (100000, 60000, 100, 5, 84), (4, 2, 1, 3, 7), (3, 2, 1, 9, 9),
              (5, 3, 1, 99, 9), (6, 4, 0, 1000, 1), (2, 1, 0, 1, 1), (1, 0, 0, 5, 4), (12, 5, 2, 9999, 10)]
    for _ in range(80):
        a = rng.randint(2, 400)
        b = rng.randint(0, a)
        c = rng.randint(0, b)
        tuples.append((a, b, c, rng.randint(1, 9999), rng.randint(1, 9999)))
    lines, want = [], []
    for a, b, c, k, j in tuples:
        for rev in (0, 1):
            lines.append("build %d %d %d %d %d %d" % (a, b, c, k, j, rev))
            try:
                want.append(oracle.build_candidate(a, b, c, k, j, bool(rev)))
            except ValueError:
                want.append(None)
    out = run(lines)
    got = [None if x == "-" else int(x, 16) for x in out]
    assert got == want
    assert sum(w is None for w in want) > 5 and sum(w is not None for w in want) > 100


def test_selfridge_parameters(run):
    """D of Selfridge's method A (or "composite": a proper factor |D|, or a
    perfect square) for every odd n < 20 000 and for large numbers of each
    kind, equal to the oracle's restatement."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import lucas
    rng = random.Random(7)
    ns = list(range(3, 20001, 2))
    ns += [rng.getrandbits(b) | 1 for b in (33, 64, 65, 500, 3000) for _ in range(10)]
    ns += [(rng.getrandbits(b) | 1) ** 2 for b in (20, 40, 300)]
    ns += [p * (rng.getrandbits(200) | 1) for p in (5, 7, 11, 13, 17, 19, 23)]
    out = run(["selfridge %s" % h(n) for n in ns])
    for n, line in zip(ns, out):
        want = lucas.selfridge_d(n)
        assert line == ("0" if want is None else "1 %d" % want), n


def test_inv_mod_lehmer(run):
    """Lehmer's extended Euclid (inv_mod): the inverse of N modulo
    2^(22 H) + 1, the Montgomery radix of the engine, for moduli of every
    transform length up to 100 000 digits, random odd moduli, and pairs with a
    common factor (no inverse)."""
    rng = random.Random(77)
    cases = []
    for H in (128, 1024, 8192, 16384):
        M = (1 << (22 * H)) + 1
        for bits in (20, 100, 22 * H - 40, 22 * H - 6):
            a = rng.getrandbits(bits) | (1 << (bits - 1)) | 1
            cases.append((a, M))
    for _ in range(40):
        M = rng.getrandbits(rng.choice([65, 128, 700, 3000])) | 1
        a = rng.randrange(1, M)
        cases.append((a, M))
    cases += [(3, 7), (1, 5), (6, 9), (10, 25), ((1 << 200) + 1, (1 << 400) - 1)]
    # a prime factor of the Fermat number 2^256 + 1 divides 2^(22*128) + 1
    cases.append((1238926361552897, (1 << 2816) + 1))
    # moduli of the Montgomery-step tests (one of them once met a Lehmer step
    # whose single-precision matrix had A = 0)
    r2 = random.Random(115)
    for abits in (1, 2, 2, 17):
        nb = 22 * 16384 - 2 - 2 * abits - r2.randrange(0, 60)
        cases.append((r2.getrandbits(nb) | 1 | (1 << (nb - 1)), (1 << (22 * 16384)) + 1))
    out = run(["inv_mod %s %s" % (h(a), h(M)) for a, M in cases])
    for (a, M), got in zip(cases, out):
        if math.gcd(a, M) != 1:
            assert got == "-", (a, M)
        else:
            assert int(got, 16) == pow(a, -1, M), (a.bit_length(), M.bit_length())
