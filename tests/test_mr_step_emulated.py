"""The engine's Montgomery step, device code and all, run on the CPU.

tests/cpp/mont_step_emul.cpp compiles prime-finder_b200/csrc/mr_device.cuh
for the host against a stand-in for the CUDA runtime (tests/cpp/emul/): one
CTA is THREADS cooperative fibers, __syncthreads a barrier over them, and the
warp ballots and shuffles exchange values through a barrier over each warp.  The
engine's own table builders (mr_tables_host.h) and modulus set-up
(bigint_host.h: N'' by Lehmer's extended Euclid) feed it.  Each result must
equal, limb for limb, Montgomery's REDC as the kernel defines it: with the
radix R' = 2^(22 H) + 1, m = -T N^-1 mod R' in [0, R') and
U = (T + m N) / R', the step leaves U * a for T = x^2 (squaring), T = x y
(general product through y's stored spectrum, the Lucas test's form) or
T = x (conversion out of Montgomery form).

This pins the arithmetic of the transforms (the zero-padded length-L product
up to 2^14; at 2^15 the cyclic and negacyclic halves of length H, the twist
by a 2H-th root of unity fused into the first and last passes), the fused
pointwise sweep, the signed CRT with its offsets, the carry-lookahead passes,
the end-around carry and the halving of V = 2U at the transform lengths 2^8,
2^9, 2^10, 2^14 and 2^15.
It does not stand in for the GPU tests: timing, memory ordering between
CTAs and the scheduler are not emulated.
"""
import os
import random
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.set_int_max_str_digits(0)
LENGTHS = (8, 9, 10, 14, 15)


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("emul") / "mont_step_emul")
    subprocess.run(["g++", "-O2", "-std=c++20", "-Wno-unknown-pragmas",
                    "-I", os.path.join(ROOT, "tests", "cpp", "emul"),
                    "-I", os.path.join(ROOT, "prime-finder_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "mont_step_emul.cpp"), "-o", exe], check=True)

    def run(lines):
        out = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True,
                             check=True, timeout=600).stdout.split()
        assert len(out) == len(lines)
        return [int(x, 16) for x in out]
    return run


def redc(logl, N, T, a=1):
    R = (1 << (22 << (logl - 1))) + 1  # R' = 2^(22 H) + 1
    m = (-T * pow(N, -1, R)) % R
    return (T + m * N) // R * a


def modulus(rng, logl, abits):
    """Odd N with R > 4 a^2 N for a of abits bits (the engine's bound)."""
    H = 1 << (logl - 1)
    nb = 22 * H - 2 - 2 * abits - rng.randrange(0, 60)
    return rng.getrandbits(nb) | 1 | (1 << (nb - 1))


@pytest.mark.parametrize("logl", LENGTHS)
def test_squaring_step(emul, logl):
    rng = random.Random(100 + logl)
    lines, want = [], []
    for a in (1, 2, 3, 65535):
        N = modulus(rng, logl, a.bit_length())
        for x in (rng.randrange(0, 4 * N), 4 * N - 1, 0, 1):
            lines.append("step %d %x %x %d" % (logl, N, x, a))
            want.append(redc(logl, N, x * x, a))
    assert emul(lines) == want


@pytest.mark.parametrize("logl", LENGTHS)
def test_general_product_and_conversion(emul, logl):
    rng = random.Random(200 + logl)
    lines, want = [], []
    for _ in range(2):
        N = modulus(rng, logl, 2)
        x, y = rng.randrange(0, 4 * N), rng.randrange(0, 4 * N)
        lines.append("mul %d %x %x %x %d" % (logl, N, x, y, 2))
        want.append(redc(logl, N, x * y, 2))
        lines.append("redc %d %x %x" % (logl, N, x))
        want.append(redc(logl, N, x))
    assert emul(lines) == want


@pytest.mark.parametrize("logl", LENGTHS)
def test_reduction_with_small_m(emul, logl):
    """REDC of T = R' - k N has m = k exactly, and of T = j N has m = R' - j:
    the step's m product returns limbs that are zero above the second, so the
    fold's test for m = lo - cM < 0 decides the result; with T = j N it is
    negative and R' is added.  k from 1 to past 2^44, j = 1, 2, 3."""
    rng = random.Random(300 + logl)
    R = (1 << (22 << (logl - 1))) + 1
    lines, want = [], []
    for _ in range(2):
        N = modulus(rng, logl, 2)
        for k in (1, 2, 3, 977, 1 << 21, (1 << 22) + 1, 1 << 43, (1 << 44) + 5, rng.getrandbits(40)):
            T = R - k * N
            if T <= 0:
                continue
            lines.append("redc %d %x %x" % (logl, N, T))
            want.append(redc(logl, N, T))
        for j in (1, 2, 3):
            lines.append("redc %d %x %x" % (logl, N, j * N))
            want.append(redc(logl, N, j * N))
    assert emul(lines) == want


def test_montgomery_ladder_equals_pow(emul):
    """A short square-and-multiply ladder in Montgomery form, fed back through
    the emulated step, ends at pow(2, e, N): the step composes as the
    persistent kernel composes it (x0 = R' mod N, one step per exponent bit,
    a final conversion)."""
    rng = random.Random(7)
    logl = 9
    H = 1 << (logl - 1)
    R = (1 << (22 * H)) + 1
    N = modulus(rng, logl, 2)
    e = rng.getrandbits(12) | (1 << 11)
    x = R % N
    for bit in bin(e)[2:]:
        x = emul(["step %d %x %x %d" % (logl, N, x, 2 if bit == "1" else 1)])[0]
    r = emul(["redc %d %x %x" % (logl, N, x)])[0]
    assert r % N == pow(2, e, N)


def test_no_out_of_bounds_access(tmp_path):
    """Built with AddressSanitizer, the emulated step touches its shared-memory
    and global buffers (exact-size host arrays here) only within bounds, for
    every form at every emulated length."""
    exe = str(tmp_path / "mont_step_emul_asan")
    cc = subprocess.run(["g++", "-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer", "-std=c++20",
                         "-Wno-unknown-pragmas",
                         "-I", os.path.join(ROOT, "tests", "cpp", "emul"),
                         "-I", os.path.join(ROOT, "prime-finder_b200", "csrc"),
                         "-I", os.path.join(ROOT, "include"),
                         os.path.join(ROOT, "tests", "cpp", "mont_step_emul.cpp"), "-o", exe],
                        capture_output=True, text=True)
    if cc.returncode != 0 and "asan" in cc.stderr.lower():
        pytest.skip("no AddressSanitizer runtime: " + cc.stderr.strip().splitlines()[-1])
    assert cc.returncode == 0, cc.stderr
    rng = random.Random(3)
    lines, want = [], []
    for logl in LENGTHS:
        N = modulus(rng, logl, 2)
        x, y = rng.randrange(0, 4 * N), rng.randrange(0, 4 * N)
        lines += ["step %d %x %x 2" % (logl, N, x), "mul %d %x %x %x 2" % (logl, N, x, y),
                  "redc %d %x %x" % (logl, N, x)]
        want += [redc(logl, N, x * x, 2), redc(logl, N, x * y, 2), redc(logl, N, x)]
    env = dict(os.environ, ASAN_OPTIONS="detect_stack_use_after_return=0:detect_leaks=0")
    r = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0 and "ERROR: AddressSanitizer" not in r.stderr, r.stderr[-2000:]
    assert [int(v, 16) for v in r.stdout.split()] == want


def test_carry_pass_and_end_around_carry(tmp_path):
    """carry_pass (three block barriers, every warp scanning the warp
    aggregates) and end_around (warp-0 ripple, full passes when the carry
    runs past limb 31) against serial carries on the host, including limbs
    of all B - 1 that make the carry run the whole length
    (tests/cpp/carry_emul.cpp)."""
    exe = str(tmp_path / "carry_emul")
    subprocess.run(["g++", "-O2", "-std=c++20", "-Wno-unknown-pragmas",
                    "-I", os.path.join(ROOT, "tests", "cpp", "emul"),
                    "-I", os.path.join(ROOT, "prime-finder_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "carry_emul.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and r.stdout.startswith("ok "), r.stdout + r.stderr
    assert int(r.stdout.split()[1]) >= 9 * 6 + 8 * 4 * 7
