"""The Phase-1 sieve kernels, device code and all, run on the CPU.

tests/cpp/sieve_emul.cpp compiles prime-finder_b200/csrc/sieve_device.cuh for
the host against the stand-in CUDA runtime of tests/cpp/emul/ (each CTA as
cooperative fibers, the CTAs of a grid one after another) and makes the
launches pfb_sieve_run and pfb_sieve_survivors make for one triple: the
prime-list split, the small-prime line records and shared-memory row tiles,
the large-prime lattice walk, and the survivor compaction.  The mask must be
bit-identical to the oracle's restatement of the reference's trial_div_cpu
(trial_div_cpu.c:32-111, any K) and the survivor list (compared through its
count and FNV-1a hash) its zero bits in k-major order; built with
AddressSanitizer, every access to the mask, the lists, the records and the
tile's shared memory must stay in bounds.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from conftest import primes_below

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "sieve_emul.cpp")
INC = ["-I", os.path.join(ROOT, "tests", "cpp", "emul"), "-I", os.path.join(ROOT, "prime-finder_b200", "csrc"),
       "-I", os.path.join(ROOT, "include")]


def _build(path, asan=False):
    flags = ["-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer"] if asan else ["-O2"]
    return subprocess.run(["g++"] + flags + ["-std=c++20", "-Wno-unknown-pragmas"] + INC + [SRC, "-o", path],
                          capture_output=True, text=True)


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("sieve_emul") / "sieve_emul")
    cc = _build(exe)
    assert cc.returncode == 0, cc.stderr
    return exe


def _run(exe, P, a, b, c, K, env=None, compact=True, unique=False):
    inp = "%d %d %d %d %d %d\n%d %s\n" % (K, a, b, c, int(compact), int(unique), len(P), " ".join(map(str, P)))
    r = subprocess.run([exe], input=inp, capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    first, second = r.stdout.split("\n")[:2]
    got = bytes.fromhex(first)
    got = np.frombuffer(got, dtype=">u4").astype("<u4").tobytes()  # words were printed big-endian
    count, h = map(int, second.split())
    return got, count, h, r.stderr


def _fnv1a64(data: bytes) -> int:
    h = 1469598103934665603
    for byte in data:
        h = ((h ^ byte) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def _check(got, count, h, P, a, b, c, K, compact=True):
    want = oracle.sieve_grid(np.asarray(P, dtype=np.uint32), a, b, c, K)
    assert got[:len(want)] == bytes(want), (a, b, c, K)
    if not compact:
        return
    bits = np.unpackbits(np.frombuffer(bytes(want), dtype=np.uint8), bitorder="little")[:K * K].reshape(K, K)
    k, j = np.nonzero(bits == 0)
    expect = (((k + 1) << 16) | (j + 1)).astype("<u4")
    assert count == len(expect)
    if len(expect) <= 200_000:
        assert h == _fnv1a64(expect.tobytes())


P5 = [p for p in primes_below(100_000).tolist() if p > 2]
CASES = [(60, 40, 20, 40), (50000, 30000, 100, 100), (181, 9, 3, 150), (101, 60, 0, 64),
         (120, 70, 30, 1000), (7, 5, 0, 100)]


@pytest.mark.parametrize("a,b,c,K", CASES)
def test_emulated_sieve_equals_oracle(emul, a, b, c, K):
    _check(*_run(emul, P5, a, b, c, K)[:3], P5, a, b, c, K)


def test_emulated_sieve_four_digit_classes(emul):
    """K = 1200: k and j of 1 to 4 digits (every digit-count class); the
    compaction's scan covers more chunks (1406) than it has threads (1024)."""
    _check(*_run(emul, P5, 50000, 30000, 100, 1200)[:3], P5, 50000, 30000, 100, 1200)


def test_emulated_sieve_full_grid(emul):
    """K = 9999, the largest grid the engine takes (the mask; the compaction
    is covered at K <= 1200)."""
    P = [p for p in primes_below(20_000).tolist() if p > 2]
    _check(*_run(emul, P, 50000, 30000, 100, 9999, compact=False)[:3], P, 50000, 30000, 100, 9999, compact=False)


def test_emulated_sieve_medium_and_large_ranges(emul):
    """Primes on both sides of the medium/large boundary (16 276 at K = 9999;
    at K = 1200 every prime is above it), in a shuffled list: the
    warp-per-prime kernel below it, the thread-per-prime kernel above, every
    digit class of k and j on one lattice walk per prime; triples with few
    classes in use (a - b = 2, a - c = 3).  Four primes near 2^31 and 2^32 check the
    Montgomery products at the top of the 32-bit range."""
    import random
    P = primes_below(1_200_000)
    pick = [int(p) for p in P[(P > 10_000) & (P < 10_400)]]
    pick += [int(p) for p in P[(P > 16_000) & (P < 16_600)]]
    pick += [int(p) for p in P[(P > 197_000) & (P < 199_500)]]
    pick += [int(p) for p in P[(P > 261_000) & (P < 264_000)]]
    pick += [int(p) for p in P[(P > 1_190_000)]][:40]
    pick += [2147483629, 2147483647, 4294967279, 4294967291]  # near 2^31 and 2^32
    random.Random(5).shuffle(pick)
    for a, b, c, K in [(50000, 30000, 100, 9999), (50000, 30000, 100, 1200), (105, 103, 102, 1200)]:
        _check(*_run(emul, pick, a, b, c, K, compact=False)[:3], pick, a, b, c, K, compact=False)


def test_line_coefficients_montgomery_and_barrett(tmp_path):
    """The large kernels' coefficients (Montgomery products on shared squaring
    chains of 10 and 10^-1) equal the small-prime set-up's (Barrett powers)
    and 128-bit powers, for primes up to just below 2^32 and exponents of
    either sign (tests/cpp/sieve_coeffs_check.cpp)."""
    exe = str(tmp_path / "coeffs")
    cc = subprocess.run(["g++", "-O2", "-std=c++20", "-Wno-unknown-pragmas"] + INC +
                        [os.path.join(ROOT, "tests", "cpp", "sieve_coeffs_check.cpp"), "-o", exe],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok "), r.stdout + r.stderr
    assert int(r.stdout.split()[1]) >= 200 * 30 * 4


def test_emulated_sieve_in_bounds(tmp_path):
    exe = str(tmp_path / "sieve_emul_asan")
    cc = _build(exe, asan=True)
    if cc.returncode != 0 and "asan" in cc.stderr.lower():
        pytest.skip("no AddressSanitizer runtime")
    assert cc.returncode == 0, cc.stderr
    env = dict(os.environ, ASAN_OPTIONS="detect_stack_use_after_return=0:detect_leaks=0")
    for a, b, c, K in [(50000, 30000, 100, 100), (181, 9, 3, 150), (120, 70, 30, 1000)]:
        got, count, surv, err = _run(exe, P5, a, b, c, K, env=env)
        assert "ERROR: AddressSanitizer" not in err
        _check(got, count, surv, P5, a, b, c, K)


def test_emulated_sieve_ignores_two_and_non_primes(emul):
    """The prime list may hold 2 (never a divisor of the odd N and rev(N)),
    and entries below 2 are ignored: the mask is the one of the odd primes."""
    P = [p for p in primes_below(20_000).tolist() if p > 2]
    base = _run(emul, P, 50000, 30000, 100, 100)
    for extra in ([2] + P, [2, 2] + P[:5] + [1, 0] + P[5:]):
        assert _run(emul, extra, 50000, 30000, 100, 100)[:3] == base[:3]


def test_emulated_unique_split_tolerates_repeats(tmp_path):
    """The allocation-free entry point's split (split_unique_kernel) lists a
    repeated value once into lists of fixed capacity: a prime list with more
    repeated small entries than the lists hold gives the mask of the list
    without repeats, and even entries are skipped.  Under AddressSanitizer,
    so an overflow of the fixed lists would show."""
    exe = str(tmp_path / "sieve_emul_asan")
    cc = _build(exe, asan=True)
    if cc.returncode != 0 and "asan" in cc.stderr.lower():
        pytest.skip("no AddressSanitizer runtime")
    assert cc.returncode == 0, cc.stderr
    env = dict(os.environ, ASAN_OPTIONS="detect_stack_use_after_return=0:detect_leaks=0")
    P = [p for p in primes_below(20_000).tolist() if p > 2]
    small = [p for p in P if p < 4096]
    noisy = [3] * 6000 + small * 3 + [4, 6, 8, 4096] + P + [11] * 100
    for K in (100, 400):
        base = _run(exe, P, 50000, 30000, 100, K, env=env)
        got = _run(exe, noisy, 50000, 30000, 100, K, env=env, unique=True)
        assert "ERROR: AddressSanitizer" not in got[3]
        assert got[:3] == base[:3]
        _check(*got[:3], P, 50000, 30000, 100, K)
