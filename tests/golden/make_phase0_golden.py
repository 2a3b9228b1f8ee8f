"""Regenerate the Phase-0 golden masks from the reference's own code.

Builds the reference's periodic table (sieve_table_build, sieve_table.c:182-243,
compiled unmodified by oracle/Makefile into oracle/_ref/libref_phase0.so) over
the odd primes below 1e4 -- the list its master uses (master.c:430) -- and
applies it (sieve_apply, sieve.c:4-22) to a fixed set of triples, writing
their 313-word masks to phase0_ref.json.  Needs 4 GB of host memory.

Usage:  python tests/golden/make_phase0_golden.py
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

TRIPLES = [(50000, 30000, 100), (50001, 30000, 100), (50000, 101, 100), (12345, 6789, 1011),
           (100000, 60000, 100), (60, 57, 2), (40, 20, 39), (99991, 12, 7), (7, 3, 1), (1, 0, 0),
           (86281, 60203, 757), (3600, 1800, 900)]


def main():
    if not os.path.exists(os.path.join(oracle.REF_DIR, "libref_phase0.so")):
        sys.exit("oracle/_ref/libref_phase0.so missing: run `make -C oracle` with the reference present")
    P = oracle.primes_below(10_000)
    t0 = time.time()
    masks = oracle.ref_phase0_masks(P, TRIPLES)
    secs = time.time() - t0
    out = {"source": "reference sieve_table_build + sieve_apply via oracle/_ref/libref_phase0.so",
           "primes": "odd primes below 1e4 (%d)" % len(P), "build_and_apply_seconds": round(secs, 1),
           "cases": [{"abc": list(t), "words_hex": m.astype("<u4").tobytes().hex()}
                     for t, m in zip(TRIPLES, masks)]}
    with open(os.path.join(HERE, "phase0_ref.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", len(TRIPLES), "masks in %.1f s" % secs)


if __name__ == "__main__":
    main()
