"""Seeded synthetic workloads of the sieve and Miller-Rabin paths.

Pure Python (no device work), shared by the benchmark and the scripts that
make the golden fixtures, so that both draw exactly the same candidates.

  uniform_batch_pairs   128 (k,j) drawn with splitmix64(seed=1), with
                        replacement, from the (k,j <= 99) sieve survivors of
                        (50000, 30000, 100): with N and rev(N), the 256
                        50 000-digit numbers of the uniform batch
  sieve_triples         (a,b,c) of the wide-grid sieve runs: a in
                        [50000, 50063], c = 100, 101, ..., b = c+1, c+1+997, ...
                        up to a-1
  uneven_tuples         512 (a,b,c,k,j,rev) with splitmix64(seed=2):
                        a ~ U[50000, 100000], c ~ U[100, 1000], b ~ U[c+1, a-1],
                        k, j ~ U[1, 9999], rev ~ U{0,1}; a tuple is drawn again
                        while a-b-lk < 2 or b-c <= lj (keeps N - 1 = 2 d with d
                        odd for both forms, and rev(N) a literal reversal)
  serving_draw          one request of the serving workload (random.Random
                        stream, same field distributions as uneven_tuples)

A draw x ~ U[lo, hi] from splitmix64 is lo + z mod (hi - lo + 1).
"""
from __future__ import annotations


def splitmix64(seed: int):
    x = seed & (2**64 - 1)
    while True:
        x = (x + 0x9E3779B97F4A7C15) & (2**64 - 1)
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
        yield z ^ (z >> 31)


def ndigits(x: int) -> int:
    return len(str(x))


def uniform_batch_pairs(survivors, n: int = 128, seed: int = 1):
    g = splitmix64(seed)
    return [tuple(survivors[next(g) % len(survivors)]) for _ in range(n)]


def sieve_triples(n: int):
    """The first n triples: c = 100, 101, ...; per c, b = c+1, c+1+997, ...
    (b <= a-1); per b, a = 50000 .. 50063."""
    out = []
    c = 100
    while len(out) < n:
        bi = 0
        while len(out) < n:
            b = c + 1 + 997 * bi
            if b > 50063 - 1:
                break
            for a in range(50000, 50064):
                if b <= a - 1 and len(out) < n:
                    out.append((a, b, c))
            bi += 1
        c += 1
    return out


def _valid(a, b, c, k, j) -> bool:
    return a - b - ndigits(k) >= 2 and b - c > ndigits(j)


def uneven_tuples(n: int = 512, seed: int = 2):
    g = splitmix64(seed)

    def u(lo, hi):
        return lo + next(g) % (hi - lo + 1)

    out = []
    while len(out) < n:
        a = u(50000, 100000)
        c = u(100, 1000)
        b = u(c + 1, a - 1)
        k = u(1, 9999)
        j = u(1, 9999)
        rev = bool(next(g) & 1)
        if _valid(a, b, c, k, j):
            out.append((a, b, c, k, j, rev))
    return out


def serving_draw(rng):
    """One serving request (a,b,c,k,j,rev) from a random.Random stream."""
    while True:
        a = rng.randint(50000, 100000)
        c = rng.randint(100, 1000)
        b = rng.randint(c + 1, a - 1)
        k, j = rng.randint(1, 9999), rng.randint(1, 9999)
        rev = bool(rng.getrandbits(1))
        if _valid(a, b, c, k, j):
            return (a, b, c, k, j, rev)
