"""The reference's BatchModCtx surface (batch_mod_ctx.cuh:132-179) on the GPU.

Compiles tests/cpp/batch_ctx_check.cpp -- a restatement of the reference's
own GMP-checked suite (correctness_tests.cuh:96-639) -- against
include/batch_mod_ctx.cuh, libpfb200.so and GMP (the declaration-only
oracle/include/gmp.h over the image's libgmp.so.10), and runs it: residue
round trips, raw squares and products against mpz_mul, modsq and modmul,
16 chained squarings, x^0xDEADBEEF against mpz_powm_ui, (N-1)^2 = 1 and
check_passed, for 512- to 332 000-bit moduli (every transform length the
engine uses for them, the 100 000-digit one included).  Every check must
pass on every modulus.
"""
import os
import subprocess

import pytest

import pfb200

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GMP = next((p for p in ("/usr/lib/x86_64-linux-gnu/libgmp.so.10", "/usr/lib64/libgmp.so.10")
            if os.path.exists(p)), None)


@pytest.fixture(scope="module")
def check(tmp_path_factory):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if GMP is None:
        pytest.skip("no libgmp runtime")
    out = str(tmp_path_factory.mktemp("cpp") / "batch_ctx_check")
    libdir = os.path.dirname(pfb200.LIB_PATH)
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "oracle", "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "batch_ctx_check.cpp"), "-o", out,
                    "-L", libdir, "-lpfb200", "-Wl,-rpath," + libdir, GMP,
                    "-L", "/usr/local/cuda/lib64", "-lcudart"], check=True)
    return out


def test_batch_mod_ctx_against_gmp(check):
    r = subprocess.run([check], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    rows = [l.split() for l in r.stdout.strip().split("\n")]
    names = {row[0] for row in rows}
    assert names == {"roundtrip", "raw_sq", "raw_mul", "modsq", "modmul", "chain16", "powm", "nm1_sq",
                     "check_passed"}
    assert {int(row[1]) for row in rows} == {512, 2048, 20000, 166000, 332000}
    for name, bits, vals, ok, bad in rows:
        assert int(bad) == 0 and int(ok) > 0, (name, bits, vals)
