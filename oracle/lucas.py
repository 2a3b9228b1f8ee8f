"""CPU restatement of the strong Lucas probable-prime test (test infrastructure).

The reference decides Phase 2 with GMP's mpz_probab_prime_p(x, 5)
(miller_rabin.c:95,107), which in GMP 6.2 and later (the image has libgmp 6.3.0)
is the Baillie-PSW test: a strong test to base 2 (mpz/millerrabin.c) followed
by a strong Lucas test with Selfridge's parameters (mpz/stronglucas.c).  GMP
is a third-party library absent from the reference tree, so the Lucas half is
restated here from its published definition (R. Baillie and S. Wagstaff,
"Lucas pseudoprimes", Math. Comp. 35 (1980); Selfridge's method A):

  D = the first of 5, -7, 9, -11, 13, ... with Jacobi (D/n) = -1
      (n composite if 1 < gcd(|D|, n) < n; squares have no such D),
  P = 1, Q = (1 - D)/4, n + 1 = 2^s d with d odd;
  n is a strong Lucas probable prime if U_d == 0 or V_(d 2^r) == 0 (mod n)
  for some 0 <= r < s.

This version walks U and V together by the binary method (the GPU engine
uses a V-only ladder), so the two share no intermediate values.  It is
checked against the published strong Lucas pseudoprimes and, through
baillie_psw(), against GMP's mpz_probab_prime_p.  Only tests/ use it.
"""
from math import gcd, isqrt


def jacobi(a: int, n: int) -> int:
    """Jacobi symbol (a / n), n odd > 0."""
    assert n > 0 and n & 1
    a %= n
    t = 1
    while a:
        while not a & 1:
            a >>= 1
            if n & 7 in (3, 5):
                t = -t
        a, n = n, a
        if a & 3 == 3 and n & 3 == 3:
            t = -t
        a %= n
    return t if n == 1 else 0


def selfridge_d(n: int):
    """Selfridge's D for odd n > 1, or None when n is found composite (a
    proper factor |D|, or a perfect square)."""
    D = 5
    tries = 0
    while True:
        tries += 1
        g = gcd(abs(D), n)
        if 1 < g < n:
            return None
        if jacobi(D, n) == -1:
            return D
        if tries == 6 and isqrt(n) ** 2 == n:
            return None
        D = -(D + 2) if D > 0 else -D + 2


def _half(x: int, n: int) -> int:
    x %= n
    return (x + n) // 2 if x & 1 else x // 2


def strong_lucas(n: int) -> int:
    """1 if odd n >= 3 is a strong Lucas probable prime, else 0."""
    if n < 3 or not n & 1:
        raise ValueError("n must be odd and >= 3")
    D = selfridge_d(n)
    if D is None:
        return 0
    Q = (1 - D) // 4
    d, s = n + 1, 0
    while not d & 1:
        d >>= 1
        s += 1
    U, V, Qk = 0, 2, 1  # k = 0
    for bit in bin(d)[2:]:
        U, V, Qk = U * V % n, (V * V - 2 * Qk) % n, Qk * Qk % n  # k -> 2k
        if bit == "1":  # k -> k + 1: U' = (P U + V)/2, V' = (D U + P V)/2
            U, V = _half(U + V, n), _half(D * U + V, n)
            Qk = Qk * Q % n
    if U == 0 or V == 0:
        return 1
    for _ in range(1, s):
        V, Qk = (V * V - 2 * Qk) % n, Qk * Qk % n
        if V == 0:
            return 1
    return 0


def strong_base2(n: int) -> int:
    d, s = n - 1, 0
    while not d & 1:
        d >>= 1
        s += 1
    x = pow(2, d, n)
    if x in (1, n - 1):
        return 1
    for _ in range(1, s):
        x = x * x % n
        if x == n - 1:
            return 1
    return 0


def baillie_psw(n: int) -> int:
    """1 probable prime / 0 composite, for any n >= 0."""
    if n < 2:
        return 0
    if not n & 1:
        return 1 if n == 2 else 0
    return 1 if strong_base2(n) and strong_lucas(n) else 0
