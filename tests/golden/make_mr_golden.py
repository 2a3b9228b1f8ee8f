"""Regenerate the full-size Miller-Rabin golden fixtures with GMP.

For every number listed below this computes, with GMP 6.3 mpz_powm (through
oracle/mr_oracle.c), the base-2 strong-test residue r = 2^d mod N
(N - 1 = 2^s d) and the verdicts, and stores a SHA-256 of r (little-endian
16-bit limbs, ceil(bits(N)/16) of them) plus its low 64 bits:

  mr_50k_first16.json     (first16) N and rev(N) of the first 16 (k,j)
                          survivors of the (50000, 30000, 100) sieve (the
                          reference's own miller_rabin_test verdicts are
                          stored beside them)
  mr_50k_survivors.json   (survivors) N and rev(N) of every survivor
                          (k,j <= 99) of that sieve: the candidates the
                          256-number uniform batch draws from
  mr_uneven_first32.json  (uneven) the first 32 of the 512 uneven-batch
                          tuples (pfb200.workloads.uneven_tuples: 50 000 -
                          100 000 digits)
  mr_uneven_first128.json (uneven128) the first 128 of those tuples (12 of
                          them at most 54 250 digits, the shorter transform
                          length); records already in mr_uneven_first32.json
                          are reused, not recomputed

Each 50 000-digit powm takes minutes of one core; the script runs a process
pool (spawn) over all cores.  Usage:
  python tests/golden/make_mr_golden.py first16|survivors|uneven|uneven128 [processes]
"""
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "prime-finder_b200"))


def residue_record(args):
    import oracle
    a, b, c, k, j, rev = args
    N = oracle.build_candidate(a, b, c, k, j, rev)
    t0 = time.time()
    s, r = oracle.strong_residue(N, 2)
    n16 = (N.bit_length() + 15) // 16
    rb = r.to_bytes(2 * n16, "little")
    verdict = 1 if (r == 1 or r == N - 1) else 0
    if not verdict and s > 1:
        verdict = oracle.strong_test(N, 2)
    return {"a": a, "b": b, "c": c, "k": k, "j": j, "rev": int(rev), "bits": N.bit_length(),
            "s": s, "sha256": hashlib.sha256(rb).hexdigest(), "low64": "%016x" % (r & (2**64 - 1)),
            "sprp2": verdict, "secs": round(time.time() - t0, 1)}


def main():
    which = sys.argv[1] if len(sys.argv) > 1 else "first16"
    sv = json.load(open(os.path.join(HERE, "sieve_50000_30000_100.json")))
    a, b, c = sv["abc"]
    pairs = [tuple(x) for x in sv["survivors_99"]]
    if which == "first16":
        pairs = pairs[:16]
    jobs = [(a, b, c, k, j, rev) for (k, j) in pairs for rev in (False, True)]
    known = {}
    if which in ("uneven", "uneven128"):
        from pfb200.workloads import uneven_tuples
        jobs = uneven_tuples(512)[:32 if which == "uneven" else 128]
        old = os.path.join(HERE, "mr_uneven_first32.json")
        if which == "uneven128" and os.path.exists(old):
            for r in json.load(open(old))["records"]:
                known[(r["a"], r["b"], r["c"], r["k"], r["j"], bool(r["rev"]))] = r
    todo = [t for t in jobs if t not in known]
    procs = int(sys.argv[2]) if len(sys.argv) > 2 else os.cpu_count()
    # longest first, so the pool's tail is short
    todo.sort(key=lambda t: -t[0])
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        for r in pool.imap_unordered(residue_record, todo, chunksize=1):
            known[(r["a"], r["b"], r["c"], r["k"], r["j"], bool(r["rev"]))] = r
            print("done", len(known), "of", len(jobs), r["a"], r["secs"], flush=True)
    recs = [known[t] for t in jobs]
    out = {"source": "GMP 6.3 mpz_powm via oracle/mr_oracle.c", "base": 2, "records": recs}
    if which not in ("uneven", "uneven128"):
        out["abc"] = [a, b, c]
    if which == "first16":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        if oracle.ref_available():
            out["ref_miller_rabin_test"] = {"%d,%d" % p: oracle.ref_miller_rabin_test(a, b, c, *p)
                                            for p in pairs}
    names = {"first16": "mr_50k_first16.json", "survivors": "mr_50k_survivors.json", "uneven": "mr_uneven_first32.json",
             "uneven128": "mr_uneven_first128.json"}
    with open(os.path.join(HERE, names[which]), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", len(recs), "records")


if __name__ == "__main__":
    main()
