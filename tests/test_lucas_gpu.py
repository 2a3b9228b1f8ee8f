"""GPU strong Lucas test and Baillie-PSW against the oracle.

pfb_mr_lucas is compared verdict for verdict with the restated strong Lucas
test (oracle/lucas.py, pinned to the published pseudoprimes and to GMP), and
pfb_mr_bpsw with GMP 6.3's mpz_probab_prime_p(n, 5) -- the call the reference's
miller_rabin_test makes (miller_rabin.c:95,107).  Known primes pin the long
transform lengths, where a restated run would take too long on the CPU: a
prime passes the strong Lucas test for every admissible D.
"""
import random

import pytest

import lucas
import oracle
import pfb200

pytestmark = pytest.mark.gpu

SLPSP = [5459, 5777, 10877, 16109, 18971, 22499, 24569, 25199, 40309, 58519, 75077, 97439, 100127]


@pytest.fixture(scope="module")
def mr():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    e = pfb200.MillerRabin(0)
    yield e
    e.close()


def test_lucas_every_small_odd_number(mr):
    ns = list(range(3, 4001, 2))
    assert mr.lucas(ns) == [lucas.strong_lucas(n) for n in ns]


def test_lucas_pseudoprimes_pass_lucas_fail_bpsw(mr):
    assert mr.lucas(SLPSP) == [1] * len(SLPSP)
    assert mr.bpsw(SLPSP) == [0] * len(SLPSP)
    spsp2 = [2047, 3277, 4033, 4681, 8321, 15841, 29341, 42799, 49141, 52633]  # base-2 strong pseudoprimes
    assert mr.bpsw(spsp2) == [0] * len(spsp2)


def _with_d(rng, D, bits, want_prime):
    while True:
        n = rng.getrandbits(bits) | (1 << (bits - 1)) | 1
        if want_prime:
            n = oracle.nextprime(n)
        if lucas.selfridge_d(n) == D:
            return n


@pytest.mark.parametrize("D", [5, -7, -11, 13, -15, 17, -19, -23])
def test_lucas_each_selfridge_class(mr, D):
    rng = random.Random(1000 + D)
    ns = [_with_d(rng, D, b, False) for b in (40, 300, 1200, 3000)]
    ns += [_with_d(rng, D, b, True) for b in (64, 400, 900)]
    assert mr.lucas(ns) == [lucas.strong_lucas(n) for n in ns]


def test_lucas_squares_factors_and_invalid(mr):
    rng = random.Random(3)
    sq = [(rng.getrandbits(b) | 1) ** 2 for b in (20, 100, 700)]
    fac = [5 * oracle.nextprime(rng.getrandbits(300)), 7 * 11 * 13 * oracle.nextprime(rng.getrandbits(200))]
    ns = sq + fac + [9, 25, 49, 3, 5, 7]
    assert mr.lucas(ns) == [lucas.strong_lucas(n) for n in ns]
    assert mr.lucas([1, 4, 1000]) == [-1, -1, -1]


def test_lucas_long_random_composite(mr):
    rng = random.Random(8)
    n = rng.getrandbits(12000) | (1 << 11999) | 1
    assert mr.lucas([n]) == [lucas.strong_lucas(n)]


def test_bpsw_equals_gmp(mr):
    rng = random.Random(29)
    ns = list(range(0, 600))
    ns += [rng.getrandbits(b) | 1 for b in (33, 64, 65, 127, 300, 1000, 2500, 6000) for _ in range(6)]
    ns += [oracle.nextprime(rng.getrandbits(b)) for b in (40, 90, 500, 1500, 3000)]
    ns += [(1 << p) - 1 for p in (89, 107, 127, 521, 607, 1279, 1281, 2203)]
    ns += [3215031751, 561 * 1105 * 1729, 3825123056546413051, 318665857834031151167461]
    assert mr.bpsw(ns) == [1 if oracle.probab_prime(n) else 0 for n in ns]


@pytest.mark.parametrize("p", [4253, 23209, 44497, 132049])
def test_lucas_mersenne_primes(mr, p):
    """M_p prime: strong Lucas passes (D = -7, -19, -11, -31: Q = 2, 5, 3, 8)."""
    assert mr.lucas([(1 << p) - 1]) == [1]


def test_lucas_mersenne_prime_long_transform(mr):
    """M_216091 (216 091 bits): the length-2^15 transforms with the spectra of
    the two NTT primes computed one after the other (D = 5, Q = -1)."""
    assert mr.lucas([(1 << 216091) - 1]) == [1]
