"""Regenerate tests/golden/sieve_k9999_full.json with the CPU oracle.

The wide-grid sieve workload tests K = 9999 grids (99 980 001 (k,j) pairs per
triple) against every odd prime below 1e8 (5 761 454 primes; 2 never divides N
or rev(N)).  The full mask of such a triple is 12.5 MB, too large to commit,
so this stores, per triple, the SHA-256 of the packed mask (ceil(K^2/8)
bytes, bit (k-1)*K + (j-1) LSB-first, 1 = eliminated), the number of
survivors and the first 64 survivors in k-major order.

The masks come from oracle/sieve_oracle.c (the restatement of the
reference's trial_div_cpu.c:32-111 for any K, itself pinned bit for bit to
the reference's own trial_div_cpu on the 100 x 100 grid).  One triple costs
about 2 000 core-seconds.

Triples: (50000, 30000, 100), the triple of the reference's own CPU run, and
three of the wide-grid enumeration (pfb200.workloads.sieve_triples): its
first, one with b = c + 1 + 7*997, and one with c = 101.

Usage: python tests/golden/make_sieve_k9999_golden.py [threads]
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "prime-finder_b200"))

K = 9999


def triples():
    from pfb200.workloads import sieve_triples
    t = sieve_triples(3264 + 64 * 40 + 64)
    # c = 100 holds 51 values of b, each with the 64 values of a
    return [(50000, 30000, 100), t[0], t[64 * 7 + 1], t[3264 + 64 * 40 + 63]]


def survivors(mask: np.ndarray, n: int):
    bits = np.unpackbits(mask, bitorder="little")[: K * K]
    idx = np.flatnonzero(bits == 0)[:n]
    return [[int(q // K) + 1, int(q % K) + 1] for q in idx]


def main():
    import oracle
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    P = oracle.primes_below(100_000_000)
    recs = []
    for (a, b, c) in triples():
        t0 = time.time()
        m = oracle.sieve_grid(P, a, b, c, K, threads=threads)
        elim = int(np.unpackbits(m, bitorder="little")[: K * K].sum())
        recs.append({"abc": [a, b, c], "sha256": hashlib.sha256(m.tobytes()).hexdigest(),
                     "survivors": K * K - elim, "first_survivors": survivors(m, 64),
                     "secs": round(time.time() - t0, 1)})
        print(recs[-1]["abc"], recs[-1]["survivors"], recs[-1]["secs"], flush=True)
    out = {"source": "oracle/sieve_oracle.c (restated trial_div_cpu), all odd primes < 1e8",
           "K": K, "primes": int(len(P)), "mask_bytes": (K * K + 7) // 8, "records": recs}
    with open(os.path.join(HERE, "sieve_k9999_full.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", len(recs), "records")


if __name__ == "__main__":
    main()
