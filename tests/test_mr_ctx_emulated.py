"""The per-operation modular context (BatchModCtx's methods), run on the CPU.

tests/cpp/ctx_emul.cpp drives the engine's host set-up, its set-up kernel
and the context's operation kernel (csrc/mr_ctx_kernels.cuh: ctx_kernel)
unchanged through the stand-in CUDA runtime of tests/cpp/emul/, one modulus
per CTA.  With R' = 2^(22 H) + 1 of the modulus' transform length, every
result must equal Python's integers: REDC(a^2) and REDC(a b) = a b R'^-1 mod N
fully reduced, the raw products a^2 and a b over n_sum = 2 n16 + 16 limbs, and
a R'^-1 mod N; at transform lengths 2^8 to 2^15 (the longest one keeps its
residue conversion's output in global memory), and once under
AddressSanitizer.
"""
import os
import random
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "ctx_emul.cpp")
INC = ["-I", os.path.join(ROOT, "tests", "cpp", "emul"), "-I", os.path.join(ROOT, "prime-finder_b200", "csrc"),
       "-I", os.path.join(ROOT, "include")]


def _build(path, asan=False):
    flags = ["-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer"] if asan else ["-O2"]
    return subprocess.run(["g++"] + flags + ["-std=c++20", "-Wno-unknown-pragmas"] + INC + [SRC, "-o", path],
                          capture_output=True, text=True)


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("ctx") / "ctx_emul")
    cc = _build(exe)
    assert cc.returncode == 0, cc.stderr
    return exe


def _run(exe, lines, env=None):
    r = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, timeout=1200,
                       env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "limb above 16 bits" not in r.stderr
    out = r.stdout.strip().split("\n")
    assert len(out) == len(lines)
    return [(int(o.split()[0]), int(o.split()[1], 16)) for o in out]


def _cases(rng, bits_list):
    cases = []
    for bits in bits_list:
        N = rng.getrandbits(bits) | (1 << (bits - 1)) | 1
        n16 = (bits + 15) // 16 + 4  # the reference pads its limb count (ntt_merge.cuh:21-24)
        a, b = rng.randrange(N), rng.randrange(N)
        for op in range(5):
            cases.append((op, n16, N, a, b))
        cases.append((0, n16, N, N - 1, 0))   # (N-1)^2 -> R^-1 mod N
        cases.append((1, n16, N, 0, b))       # zero operand
    return cases


def _want(op, n16, N, a, b, logl):
    R = (1 << (22 * (1 << (logl - 1)))) + 1
    ri = pow(R, -1, N)
    if op == 0:
        return a * a * ri % N
    if op == 1:
        return a * b * ri % N
    if op == 2:
        return a * a
    if op == 3:
        return a * b
    return a * ri % N


def _check(res, cases):
    for (op, n16, N, a, b), (logl, got) in zip(cases, res):
        assert logl > 0
        assert 22 * (1 << (logl - 1)) >= N.bit_length() + 6
        assert got == _want(op, n16, N, a, b, logl), (op, N.bit_length(), logl)


def test_ctx_ops_short_lengths(emul):
    rng = random.Random(31)
    cases = _cases(rng, [17, 100, 1000, 2790, 2900, 5000, 11000])
    _check(_run(emul, ["%d %d %x %x %x" % c for c in cases]), cases)


def test_ctx_ops_long_lengths(emul):
    """Transform lengths 2^14 (both primes on chip) and 2^15 (one prime's
    coefficients spilled to global memory): 50 000 and 100 000 digits."""
    rng = random.Random(32)
    cases = _cases(rng, [166000, 332000])
    _check(_run(emul, ["%d %d %x %x %x" % c for c in cases]), cases)


def test_ctx_in_bounds(tmp_path):
    exe = str(tmp_path / "ctx_emul_asan")
    cc = _build(exe, asan=True)
    if cc.returncode != 0 and "asan" in cc.stderr.lower():
        pytest.skip("no AddressSanitizer runtime")
    assert cc.returncode == 0, cc.stderr
    env = dict(os.environ, ASAN_OPTIONS="detect_stack_use_after_return=0:detect_leaks=0")
    rng = random.Random(33)
    cases = _cases(rng, [300, 3000])
    _check(_run(exe, ["%d %d %x %x %x" % c for c in cases], env=env), cases)
