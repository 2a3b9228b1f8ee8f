"""Sieve -> test pipeline (pfb_pipeline_run) against the oracle.

The expected records come from the oracle's restated sieve (trial_div_cpu for
any K) and GMP's mpz_probab_prime_p(x, 5) on N and rev(N) exactly as the
reference's miller_rabin_test combines them (miller_rabin.c:76-118), and, when
the reference's own miller_rabin.c is built under oracle/_ref, from that
function itself.
"""
import json
import os

import numpy as np
import pytest

import oracle
import pfb200
from conftest import primes_below

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def engines():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    sv = pfb200.Sieve(primes_below(100_000))
    mr = pfb200.MillerRabin(0)
    yield sv, mr
    sv.close()
    mr.close()


def _expected(P, abc, K, pre=None):
    out = []
    blk = pfb200.mask_bytes(K)  # device block: 4 * ceil(K^2 / 32) bytes
    for t, (a, b, c) in enumerate(abc):
        m = oracle.sieve_grid(P, a, b, c, K)  # ceil(K^2 / 8) bytes
        if pre is not None:
            m = m | pre[t * blk:t * blk + len(m)]
        bits = np.unpackbits(m, bitorder="little")[:K * K].reshape(K, K)
        for k, j in zip(*np.nonzero(bits == 0)):
            k, j = int(k) + 1, int(j) + 1
            if oracle.probab_prime(oracle.build_candidate(a, b, c, k, j, False)) == 0:
                r = 0
            else:
                r = 2 if oracle.probab_prime(oracle.build_candidate(a, b, c, k, j, True)) else 1
            out.append((a, b, c, k, j, r))
    return out


ABC = [(60, 40, 20), (81, 61, 27), (120, 70, 30), (150, 100, 2), (101, 60, 0), (181, 9, 3)]


def test_pipeline_matches_oracle(engines):
    sv, mr = engines
    K = 40
    recs, st = pfb200.pipeline_run(sv, mr, ABC, K, triples_per_sieve=2)
    want = _expected(primes_below(100_000), ABC, K)
    assert recs == want
    assert st["survivors"] == len(want) and st["triples"] == len(ABC)
    assert st["n_prp"] == sum(1 for r in want if r[5] > 0)
    assert st["both_prp"] == sum(1 for r in want if r[5] == 2)
    assert st["n_prp"] > 0 and st["rev_tested"] > 0 and st["both_prp"] >= 3  # every code occurs
    if oracle.ref_available():  # the reference's own miller_rabin_test (k, j < 100)
        for a, b, c, k, j, r in recs:
            assert oracle.ref_miller_rabin_test(a, b, c, k, j) == r, (a, b, c, k, j)


def test_pipeline_pre_mask_and_capacity(engines):
    sv, mr = engines
    K = 25
    abc = ABC[:2]
    blk = pfb200.mask_bytes(K)
    rng = np.random.default_rng(4)
    pre = (rng.random(blk * len(abc)) < 0.3).astype(np.uint8) * rng.integers(1, 256, blk * len(abc), dtype=np.uint8)
    recs, _ = pfb200.pipeline_run(sv, mr, abc, K, pre_mask=pre)
    assert recs == _expected(primes_below(100_000), abc, K, pre)
    with pytest.raises(pfb200.PfbError) as ei:
        pfb200.pipeline_run(sv, mr, abc, K, cap=1)
    assert ei.value.code == -4


def test_pipeline_50000_30000_100_corner(primes_1e8):
    """(50000, 30000, 100) on the 20 x 20 corner with every prime below 1e8:
    the survivors are the reference's, and every 50 000-digit N is composite
    (the reference's miller_rabin_test returns 0 for all of them)."""
    g = json.load(open(os.path.join(GOLD, "sieve_50000_30000_100.json")))
    sv = pfb200.Sieve(primes_1e8)
    mr = pfb200.MillerRabin(0)
    recs, st = pfb200.pipeline_run(sv, mr, [tuple(g["abc"])], 20)
    want = [(50000, 30000, 100, k, j, 0) for k, j in g["survivors_99"] if k <= 20 and j <= 20]
    assert recs == want and len(want) == 3
    sv.close()
    mr.close()
