"""The Phase-0 kernels, device code and all, run on the CPU.

tests/cpp/phase0_emul.cpp compiles prime-finder_b200/csrc/phase0_device.cuh
for the host against the stand-in CUDA runtime of tests/cpp/emul/ and runs
build_kernel over the whole table and apply_kernel per triple, with the table
entries pfb_phase0_create builds.  The primes are a set with small
multiplicative orders of 10 (about 13 000 masks instead of the 3.2 M of the
primes below 10^4), so every code path of the mask construction runs at CPU
speed.  The masks must equal the restated Phase 0 (oracle/phase0.py) and,
where the reference was compiled here, its own sieve_table_build +
sieve_apply (sieve_table.c:93-243); built with AddressSanitizer, every
access must stay in bounds.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
import phase0

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "phase0_emul.cpp")
INC = ["-I", os.path.join(ROOT, "tests", "cpp", "emul"), "-I", os.path.join(ROOT, "prime-finder_b200", "csrc"),
       "-I", os.path.join(ROOT, "include")]
# ord_p(10): 1, 6, 2, 6, 16, 15, 3, 5, 13, 8, 13, 4 (and 97: 96 > 64, not tabled)
PRIMES = [3, 7, 11, 13, 17, 31, 37, 41, 53, 73, 79, 101, 97]


def _triples():
    rng = np.random.default_rng(5)
    abc = [(50000, 30000, 100), (60, 40, 20), (5, 3, 0), (1, 0, 0)]
    abc += [(int(a), int(rng.integers(0, a)), int(rng.integers(0, 1000))) for a in rng.integers(1000, 200000, 8)]
    return abc


def _run(exe, abc, env=None):
    inp = "%d %s\n%d %s\n" % (len(PRIMES), " ".join(map(str, PRIMES)), len(abc),
                              " ".join("%d %d %d" % t for t in abc))
    r = subprocess.run([exe], input=inp, capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [np.frombuffer(bytes.fromhex(line), dtype=">u4").astype(np.uint32) for line in r.stdout.split()], r.stderr


def _build(path, asan=False):
    flags = ["-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer"] if asan else ["-O2"]
    return subprocess.run(["g++"] + flags + ["-std=c++20", "-Wno-unknown-pragmas"] + INC + [SRC, "-o", path],
                          capture_output=True, text=True)


def test_emulated_phase0_equals_restatement_and_reference(tmp_path):
    exe = str(tmp_path / "phase0_emul")
    cc = _build(exe)
    assert cc.returncode == 0, cc.stderr
    abc = _triples()
    got, _ = _run(exe, abc)
    P = np.array(PRIMES, dtype=np.uint32)
    for t, m in zip(abc, got):
        assert (m == phase0.phase0_mask(P, *t)).all(), t
    if os.path.exists(os.path.join(oracle.REF_DIR, "libref_phase0.so")):
        want = oracle.ref_phase0_masks(P, abc)
        for t, m, w in zip(abc, got, want):
            assert (m == w).all(), t
    assert sum(int(x).bit_count() for m in got for x in m) > 10_000  # the masks are not trivially empty


def test_emulated_phase0_in_bounds(tmp_path):
    exe = str(tmp_path / "phase0_emul_asan")
    cc = _build(exe, asan=True)
    if cc.returncode != 0 and "asan" in cc.stderr.lower():
        pytest.skip("no AddressSanitizer runtime")
    assert cc.returncode == 0, cc.stderr
    env = dict(os.environ, ASAN_OPTIONS="detect_stack_use_after_return=0:detect_leaks=0")
    abc = _triples()[:4]
    got, err = _run(exe, abc, env=env)
    assert "ERROR: AddressSanitizer" not in err
    P = np.array(PRIMES, dtype=np.uint32)
    for t, m in zip(abc, got):
        assert (m == phase0.phase0_mask(P, *t)).all(), t
