"""Regenerate the golden sieve fixtures from the reference's own CPU code.

Runs the reference's unmodified trial_div_cpu() (compiled by oracle/Makefile
into oracle/_ref/libref_sieve.so from the reference sources) and writes:

  sieve_ref_kat.json   - 313-word masks for the prime list of tests/test_gpu.c
                         (3..97) at the (a,b,c) of tests/test_gpu.c:169-172 and
                         tests/test_sieve.c:78-80
  sieve_50000_30000_100.json   - the 100 x 100 mask at (a,b,c) = (50000, 30000, 100)
                         over every odd prime below 1e8, with its survivors

Usage:  python tests/golden/make_golden.py          (needs oracle/_ref built)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

KAT_PRIMES = [3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73,
              79, 83, 89, 97]
KAT_ABC = [(15, 8, 3), (20, 10, 5), (25, 12, 6), (12, 6, 3), (30, 15, 7)]


def words_hex(bits: np.ndarray) -> str:
    return bits.astype("<u4").tobytes().hex()


def survivors(bits: np.ndarray, K: int = 100):
    m = np.unpackbits(bits.astype("<u4").view(np.uint8), bitorder="little")[: K * K].reshape(K, K)
    return [[k + 1, j + 1] for k in range(K) for j in range(K) if not m[k, j]]


def main():
    if not oracle.ref_available():
        sys.exit("oracle/_ref/libref_sieve.so missing: run `make -C oracle` with the reference present")
    kat = []
    p = np.array(KAT_PRIMES, dtype=np.uint32)
    for a, b, c in KAT_ABC:
        bits = oracle.ref_trial_div_cpu(p, a, b, c)
        kat.append({"abc": [a, b, c], "words_hex": words_hex(bits)})
    with open(os.path.join(HERE, "sieve_ref_kat.json"), "w") as f:
        json.dump({"source": "reference trial_div_cpu.c via oracle/_ref/libref_sieve.so",
                   "primes": KAT_PRIMES, "cases": kat}, f, indent=1)

    P = oracle.primes_below(100_000_000)
    a, b, c = 50000, 30000, 100
    bits = oracle.ref_trial_div_cpu(P, a, b, c)
    surv = survivors(bits)
    sub = [s for s in surv if s[0] <= 99 and s[1] <= 99]
    with open(os.path.join(HERE, "sieve_50000_30000_100.json"), "w") as f:
        json.dump({"source": "reference trial_div_cpu.c via oracle/_ref/libref_sieve.so",
                   "primes": "odd primes below 1e8 (%d)" % len(P), "n_primes": int(len(P)),
                   "abc": [a, b, c], "words_hex": words_hex(bits),
                   "n_survivors_100": len(surv), "n_survivors_99": len(sub),
                   "survivors_99": sub}, f, indent=1)
    print("wrote", len(kat), "KAT cases;", len(surv), "(50000,30000,100) survivors (", len(sub), "on 99x99 )")


if __name__ == "__main__":
    main()
