"""The Phase-0 restatement (oracle/phase0.py) pinned to the reference's own
sieve_table_build + sieve_apply (tests/golden/phase0_ref.json, made by
tests/golden/make_phase0_golden.py from the reference's unmodified code)."""
import json
import os

import numpy as np

import oracle
import phase0

GOLD = os.path.join(os.path.dirname(__file__), "golden", "phase0_ref.json")


def test_tabled_primes_below_1e4():
    t = phase0.tabled(oracle.primes_below(10_000))
    assert len(t) == 62 and t[0] == (3, 1) and (9901, 12) in t
    assert sum(L ** 3 for _, L in t) == 3_208_136


def test_restatement_equals_reference_masks():
    g = json.load(open(GOLD))
    P = oracle.primes_below(10_000)
    for case in g["cases"]:
        a, b, c = case["abc"]
        want = np.frombuffer(bytes.fromhex(case["words_hex"]), dtype="<u4")
        assert (phase0.phase0_mask(P, a, b, c) == want).all(), case["abc"]


def test_phase0_bits_are_trial_division_bits():
    # where every exponent is non-negative, Phase 0 eliminates a subset of what
    # trial division by the same primes eliminates (it skips the primes whose
    # ord_p(10)^3 > 2^18)
    P = oracle.primes_below(10_000)
    for a, b, c in [(50000, 30000, 100), (12345, 6789, 1011)]:
        p0 = phase0.phase0_mask(P, a, b, c)
        td = oracle.ref_trial_div_cpu(P, a, b, c) if oracle.ref_available() else None
        if td is not None:
            assert not (p0 & ~td).any()
