"""The strong Lucas restatement (oracle/lucas.py) pinned to published values
and to GMP: its pseudoprimes below 130 000 are the published strong Lucas
pseudoprimes (Selfridge's parameters), and its Baillie-PSW equals GMP 6.3's
mpz_probab_prime_p(n, 5) verdict on every n below 20 000 and on random and
structured large numbers."""
import random

import lucas
import oracle

# strong Lucas pseudoprimes with Selfridge's parameters below 130 000
# (Baillie and Wagstaff 1980; OEIS A217255)
SLPSP = [5459, 5777, 10877, 16109, 18971, 22499, 24569, 25199, 40309, 58519, 75077, 97439, 100127,
         113573, 115639]


def _is_prime(n):
    if n < 2:
        return False
    i = 2
    while i * i <= n:
        if n % i == 0:
            return False
        i += 1
    return True


def test_jacobi_small():
    for n in range(1, 200, 2):
        for a in range(-50, 50):
            # Euler's criterion for odd primes
            if _is_prime(n) and n > 2 and a % n:
                assert lucas.jacobi(a, n) == (1 if pow(a % n, (n - 1) // 2, n) == 1 else -1)


def test_strong_lucas_pseudoprimes_match_published_list():
    got = [n for n in range(3, 130_000, 2) if lucas.strong_lucas(n) and not _is_prime(n)]
    assert got == SLPSP


def test_primes_pass_and_squares_fail():
    assert all(lucas.strong_lucas(p) for p in range(3, 5000, 2) if _is_prime(p))
    assert not any(lucas.strong_lucas(m * m) for m in range(3, 400, 2))


def test_baillie_psw_equals_gmp():
    for n in range(20_000):
        assert lucas.baillie_psw(n) == (1 if oracle.probab_prime(n) else 0), n
    rng = random.Random(17)
    nums = [rng.getrandbits(b) | 1 for b in (64, 65, 100, 300, 521, 1000, 2000) for _ in range(20)]
    nums += [oracle.nextprime(rng.getrandbits(b)) for b in (70, 200, 700, 1500)]
    nums += [(1 << p) - 1 for p in (521, 607, 1279, 1281)]
    nums += [3215031751, 2047 * 4033, 561 * 1105, 25326001, 3825123056546413051]
    for n in nums:
        assert lucas.baillie_psw(n) == (1 if oracle.probab_prime(n) else 0), n
