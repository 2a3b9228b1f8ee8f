"""The reference's C++ Miller-Rabin surface and miller_rabin_test, used from C++.

Compiles tests/cpp/mr_api_demo.cpp against include/ and libpfb200.so (the
way bench_mr_gpu.cu and worker.c would link), runs it, and checks:
  * Mersenne primes M521/M607/M1279 pass all 16 DEFAULT_WITNESSES through
    BatchModCtx + gpu_miller_rabin_s1 (correctness_tests.cuh:762-834);
  * miller_rabin_test returns what the reference's own miller_rabin_test
    (oracle/_ref, GMP BPSW) returns, on small (a,b,c,k,j) and on
    tests/test_phase2.c's grid.
"""
import os
import random
import subprocess

import pytest

import oracle
import pfb200

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    out = str(tmp_path_factory.mktemp("cpp") / "mr_api_demo")
    libdir = os.path.dirname(pfb200.LIB_PATH)
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "mr_api_demo.cpp"), "-o", out,
                    "-L", libdir, "-lpfb200", "-Wl,-rpath," + libdir], check=True)
    return out


def test_cpp_surface_and_miller_rabin_test(demo):
    rng = random.Random(4)
    cases = [(4, 2, 1, k, j) for k in range(1, 6) for j in range(1, 6)]  # tests/test_phase2.c:46-72
    while len(cases) < 60:
        a = rng.randint(8, 40)
        b = rng.randint(4, a - 4)
        c = rng.randint(1, b - 2)
        cases.append((a, b, c, rng.randint(1, 99), rng.randint(1, 9)))
    args = [str(x) for cs in cases for x in cs]
    out = subprocess.run([demo] + args, check=True, capture_output=True, text=True).stdout.split("\n")
    mers = [l.split() for l in out if l.startswith("mersenne")]
    assert [int(m[2]) for m in mers] == [1, 1, 1]
    got = {tuple(int(x) for x in l.split()[1:6]): int(l.split()[6]) for l in out if l.startswith("mrt")}
    for cs in cases:
        want = oracle.ref_miller_rabin_test(*cs) if oracle.ref_available() else None
        N = oracle.build_candidate(*cs, False)
        if want is None:
            want = 0 if not oracle.probab_prime(N, 5) else (
                2 if oracle.probab_prime(oracle.build_candidate(*cs, True), 5) else 1)
        assert got[cs] == want, cs
