"""The seeded workload generators: deterministic, and the uneven-batch tuples
respect the constraints that keep N - 1 = 2 d (d odd) and rev(N) literal."""
import random
import sys

import pfb200
from pfb200 import workloads as W

sys.set_int_max_str_digits(0)


def test_splitmix64_known_values():
    # splitmix64 from seed 0: the published first outputs of the generator
    g = W.splitmix64(0)
    assert [next(g) for _ in range(3)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_uniform_batch_is_deterministic():
    surv = [(k, j) for k in range(1, 11) for j in range(1, 12)]
    a = W.uniform_batch_pairs(surv)
    assert a == W.uniform_batch_pairs(surv) and len(a) == 128
    assert all(p in surv for p in a)


def test_sieve_triples_enumeration():
    t = W.sieve_triples(200)
    assert t[0] == (50000, 101, 100) and t[63] == (50063, 101, 100) and t[64] == (50000, 1098, 100)
    assert all(c == 100 and c < b < a for a, b, c in t)


def test_uneven_tuples_constraints():
    t = W.uneven_tuples(512)
    assert t == W.uneven_tuples(512) and len(t) == 512
    for a, b, c, k, j, rev in t:
        assert 50000 <= a <= 100000 and 100 <= c <= 1000 and c < b < a and 1 <= k <= 9999 and 1 <= j <= 9999
        assert a - b - len(str(k)) >= 2 and b - c > len(str(j))
    assert {r for *_, r in t} == {False, True}
    for tup in t[:4]:
        N = pfb200.build_candidate(*tup)
        assert N % 4 == 3  # N - 1 = 2 d with d odd
        assert len(str(N)) == tup[0]


def test_serving_draw_constraints():
    rng = random.Random(3)
    for _ in range(50):
        a, b, c, k, j, rev = W.serving_draw(rng)
        assert a - b - len(str(k)) >= 2 and b - c > len(str(j))


def test_sieve_triples_continue_past_the_first_c():
    t = W.sieve_triples(5000)
    assert len(t) == 5000 and len(set(t)) == 5000
    assert all(50000 <= a <= 50063 and c < b <= a - 1 for a, b, c in t)
    assert t[3264] == (50000, 102, 101)
