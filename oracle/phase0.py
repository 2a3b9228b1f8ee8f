"""CPU restatement of the reference's Phase-0 periodic sieve table (test
infrastructure; only tests/ use it).

Follows sieve_table.c:19-35 (ord_p(10)), :93-178 (fill_prime_bitmask) and
sieve.c:4-22 (sieve_apply): a prime p >= 3 with L = ord_p(10) and L^3 <= 2^18
contributes, for (a, b, c), the 100 x 100 mask of the residue triple
(a mod L, b mod L, c mod L); bit (k-1)*100 + (j-1) set = eliminated.  Only the
one mask each prime contributes is computed here (the reference tabulates all
L^3 of them).
"""
from typing import List, Sequence

import numpy as np

WORDS = 313
MAX_ENTRIES = 1 << 18


def mult_order10(p: int) -> int:
    """ord_p(10), 0 when p divides 10."""
    if 10 % p == 0:
        return 0
    x, r = 10 % p, 1
    while x != 1:
        x = x * 10 % p
        r += 1
    return r


def tabled(primes: Sequence[int]) -> List[tuple]:
    out = []
    for p in primes:
        p = int(p)
        if p < 3:
            continue
        L = mult_order10(p)
        if L and L ** 3 <= MAX_ENTRIES:
            out.append((p, L))
    return out


def cell_mask(p: int, L: int, ra: int, rb: int, rc: int) -> np.ndarray:
    """The 313-word mask of sieve_table.c:93-178 for one residue triple."""
    bits = np.zeros(WORDS * 32, dtype=bool)
    P = [pow(10, r, p) for r in range(L)]
    I = [pow(P[r], p - 2, p) for r in range(L)]
    for k in range(1, 101):  # N form
        num = (P[ra] - k * P[rb] % p - 1 + 2 * p) % p
        j = num * I[rc] % p or p
        while j <= 100:
            bits[(k - 1) * 100 + j - 1] = True
            j += p
    c1 = I[ra] * P[(rc + 1) % L] % p
    c2 = I[ra] * P[(rc + 2) % L] % p
    r3 = P[ra] * I[(rc + 3) % L] % p
    for k in range(1, 101):  # rev form
        lk = 1 if k < 10 else 2 if k < 100 else 3
        rk = int(str(k).zfill(lk)[::-1])
        rb_rev = P[ra] * I[(rb + lk) % L] % p
        base = (P[ra] - rk * rb_rev % p - 1 + 2 * p) % p
        if c1:
            j = base * c1 % p or p
            while j <= 9:
                bits[(k - 1) * 100 + j - 1] = True
                j += p
        if c2:
            rj = base * c2 % p or p
            while rj <= 99:
                j = rj * 10 if rj <= 9 else ((rj % 10) * 10 + rj // 10 if rj % 10 else -1)
                if 10 <= j <= 99:
                    bits[(k - 1) * 100 + j - 1] = True
                rj += p
        if r3 and r3 == base:
            bits[(k - 1) * 100 + 99] = True
    return np.packbits(bits, bitorder="little").view("<u4").copy()


def phase0_mask(primes: Sequence[int], a: int, b: int, c: int) -> np.ndarray:
    """sieve_apply for one triple: the OR of every tabled prime's mask."""
    m = np.zeros(WORDS, dtype=np.uint32)
    for p, L in tabled(primes):
        m |= cell_mask(p, L, a % L, b % L, c % L)
    return m
