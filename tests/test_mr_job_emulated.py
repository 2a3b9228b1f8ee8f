"""Whole strong tests and strong Lucas tests of the engine, run on the CPU.

tests/cpp/mr_job_emul.cpp drives the engine's own host set-up
(csrc/mr_prep_host.h: host_prep), set-up kernel and persistent scheduler
(csrc/mr_kernels.cuh: prep_kernel, persist_kernel -> run_job / run_lucas)
unchanged, one candidate per CTA, through the stand-in CUDA runtime of
tests/cpp/emul/.  Verdicts and residues must equal GMP's (mpz_powm, the
strong test of the reference's oracle) and the restated strong Lucas test
(oracle/lucas.py), including the base-2 strong pseudoprimes, the strong
Lucas pseudoprimes, s > 1 and the numbers the host decides on its own.
"""
import os
import random
import subprocess

import pytest

import lucas
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("mr_job") / "mr_job_emul")
    subprocess.run(["g++", "-O2", "-std=c++20", "-Wno-unknown-pragmas",
                    "-I", os.path.join(ROOT, "tests", "cpp", "emul"),
                    "-I", os.path.join(ROOT, "prime-finder_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "mr_job_emul.cpp"), "-o", exe], check=True)

    def run(lines):
        out = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True,
                             timeout=900).stdout.strip().split("\n")
        assert len(out) == len(lines)
        return out
    return run


def test_strong_test_verdicts_and_residues(emul):
    rng = random.Random(11)
    ns = [3, 5, 7, 9, 15, 561, 1105, 2047, 3277, 4033, 4681, 8321, 65537, 1000001, 1000003,
          (1 << 61) - 1, (1 << 89) - 1, 2 ** 64 + 13]
    ns += [rng.getrandbits(b) | 1 | (1 << (b - 1)) for b in (24, 33, 64, 100)]
    out = emul(["1 2 %x" % n for n in ns])
    for n, line in zip(ns, out):
        v, r = line.split()
        s, res = oracle.strong_residue(n, 2)
        assert (int(v), int(r, 16)) == (oracle.strong_test(n, 2), res), n


def test_other_bases_and_rejections(emul):
    ns = [(3, 1000003), (7, 3215031751), (65535, 1000033)]
    out = emul(["1 %d %x" % (a, n) for a, n in ns] + ["1 2 %x" % n for n in (1, 4, 100)])
    for (a, n), line in zip(ns, out[:3]):
        v, r = line.split()
        assert (int(v), int(r, 16)) == (oracle.strong_test(n, a), oracle.strong_residue(n, a)[1]), (a, n)
    assert [line.split()[0] for line in out[3:]] == ["-1", "-1", "-1"]


def test_strong_lucas_verdicts(emul):
    rng = random.Random(12)
    ns = [5459, 5777, 10877, 16109, 18971, 3, 5, 7, 11, 13, 25, 49, 1000003, 1000001, (1 << 61) - 1]
    ns += [rng.getrandbits(b) | 1 | (1 << (b - 1)) for b in (30, 50, 70)]
    out = emul(["2 2 %x" % n for n in ns])
    assert [int(v) for v in out] == [lucas.strong_lucas(n) for n in ns]


def _with_d(rng, D, bits, want_prime):
    while True:
        n = rng.getrandbits(bits) | (1 << (bits - 1)) | 1
        if want_prime:
            n = oracle.nextprime(n)
        if lucas.selfridge_d(n) == D:
            return n


@pytest.mark.parametrize("D", [5, -7, -11, 13, -15, 17, -19, -23])
def test_strong_lucas_each_selfridge_class(emul, D):
    """One composite and one prime per Selfridge class D (Q = (1 - D) / 4:
    -1, 2, 3, -3, 4, -4, 5, 6), through the emulated Lucas ladder."""
    rng = random.Random(2000 + D)
    ns = [_with_d(rng, D, 90, False), _with_d(rng, D, 120, True)]
    assert [int(v) for v in emul(["2 2 %x" % n for n in ns])] == [lucas.strong_lucas(n) for n in ns]
