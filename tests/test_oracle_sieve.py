"""CPU checks of the sieve oracle: pinned to the reference's own outputs.

The restatement in oracle/sieve_oracle.c must reproduce the reference's
trial_div_cpu.c (golden fixtures generated from the reference by
tests/golden/make_golden.py) and the definitional brute force of
tests/test_gpu.c:31-73 on every grid size.
"""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import primes_below

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _words(h: str) -> np.ndarray:
    return np.frombuffer(bytes.fromhex(h), dtype="<u4").copy()


def test_restatement_matches_reference_kat():
    g = json.load(open(os.path.join(GOLD, "sieve_ref_kat.json")))
    p = np.array(g["primes"], dtype=np.uint32)
    for case in g["cases"]:
        a, b, c = case["abc"]
        mine = oracle.sieve_grid(p, a, b, c, 100, threads=1)
        ref = _words(case["words_hex"]).view(np.uint8)[:1250]
        assert (mine == ref).all(), case["abc"]


def test_brute_force_matches_reference_kat():
    g = json.load(open(os.path.join(GOLD, "sieve_ref_kat.json")))
    p = np.array(g["primes"], dtype=np.uint32)
    for case in g["cases"]:
        a, b, c = case["abc"]
        assert (oracle.sieve_brute(p, a, b, c, 100) ==
                _words(case["words_hex"]).view(np.uint8)[:1250]).all()


@pytest.mark.parametrize("K", [1, 9, 10, 11, 37, 99, 100, 101, 150])
def test_restatement_equals_brute_force(K):
    rng = np.random.default_rng(K)
    P = primes_below(5000)
    for _ in range(3):
        p = np.sort(rng.choice(P, size=40, replace=False)).astype(np.uint32)
        p = np.concatenate([np.array([3, 5, 7], np.uint32), p])
        a = int(rng.integers(8, 400))
        b = int(rng.integers(1, a))
        c = int(rng.integers(0, b + 3))
        m1 = oracle.sieve_grid(p, a, b, c, K, threads=2)
        m2 = oracle.sieve_brute(p, a, b, c, K)
        assert (m1 == m2).all(), (K, a, b, c)


def test_negative_rev_exponents():
    # b close to a: a-b-lk < 0 for some digit classes (rev terms skipped, as the reference does)
    p = primes_below(3000)
    for a, b, c in [(6, 5, 1), (7, 4, 3), (9, 8, 8), (12, 9, 0)]:
        assert (oracle.sieve_grid(p, a, b, c, 120, threads=2) ==
                oracle.sieve_brute(p, a, b, c, 120)).all()


def test_50000_30000_100_golden_against_restatement():
    g = json.load(open(os.path.join(GOLD, "sieve_50000_30000_100.json")))
    P = primes_below(100_000_000)
    assert len(P) == g["n_primes"] == 5761454
    a, b, c = g["abc"]
    mine = oracle.sieve_grid(P, a, b, c, 100)
    assert (mine == _words(g["words_hex"]).view(np.uint8)[:1250]).all()


def test_prime_generator():
    P = primes_below(1000)
    assert P[0] == 3 and P[-1] == 997 and len(P) == 167
    assert len(primes_below(100_000_000)) == 5761454
