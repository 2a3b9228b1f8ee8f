"""bench.py's bookkeeping on the CPU: the reference-structure work count the
roofline divides by, and the small kernel cases used for ncu captures."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_work_count():
    """M(L) = 2 (6 (L/2) log2 L + 3 L) modmuls x 3 INT32 multiplies per
    squaring: 9.44 M at 50 000 digits (L = 2^15 in the reference's 16-bit
    limbs, ntt_merge.cuh:21-24) and 20.05 M at 100 000 digits (L = 2^16)."""
    assert bench.ref_modmuls_per_squaring(50000) * bench.SQ_PER_MODMUL == 9437184
    assert bench.ref_modmuls_per_squaring(100000) * bench.SQ_PER_MODMUL == 20054016
    L = 1 << 15
    assert bench.ref_modmuls_per_squaring(50000) == 2 * (6 * (L // 2) * 15 + 3 * L)


def test_mr_cases_are_eight_candidates():
    for name, (abc, pairs) in bench.MR_CASES.items():
        a, b, c = abc
        assert c < b < a
        if pairs is not None:
            assert len(pairs) == 4  # N and rev(N) of each: 8 candidates, one CTA each


def test_sieve_input_primes():
    P = bench.odd_primes_below(1_000_000)
    assert len(P) == 78497 and P[0] == 3 and P[-1] == 999983  # pi(10^6) = 78498, less the prime 2
    assert len(bench.odd_primes_below(100)) == 24
