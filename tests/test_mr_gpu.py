"""GPU parity of the Miller-Rabin engine against GMP (the oracle).

Mirrors miller_rabin_gpu/correctness_tests.cuh: modular powers against
mpz_powm (:578-639 uses x^0xDEADBEEF), Mersenne primes M521/M607/M1279
through all 16 default witnesses (:762-834), primes with s = 1 and s > 1
generated by mpz_nextprime above 2^512 (:842-1031), plus random composites.
Residues are compared word for word; verdicts bit for bit.
"""
import hashlib
import json
import os
import random

import numpy as np
import pytest

import oracle
import pfb200

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
WITNESSES = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53]  # runner.cuh:15-16


@pytest.fixture(scope="module")
def mr():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    e = pfb200.MillerRabin(0)
    yield e
    e.close()


def _gmp_powm(base, E, N):
    bl = oracle.int_to_limbs(base, 1)
    el = oracle.int_to_limbs(E, (E.bit_length() + 15) // 16)
    n16 = (N.bit_length() + 15) // 16
    nl = oracle.int_to_limbs(N, n16)
    out = np.zeros(n16, dtype=np.uint16)
    L = oracle.lib()
    L.oracle_powm(oracle._ptr(bl, oracle.C.c_uint16), 1, oracle._ptr(el, oracle.C.c_uint16), len(el),
                  oracle._ptr(nl, oracle.C.c_uint16), n16, oracle._ptr(out, oracle.C.c_uint16))
    return oracle.limbs_to_int(out)


def test_powm_small_vs_gmp(mr):
    rng = random.Random(0xDEADBEEF)
    Ns, Es = [], []
    for bits in (3, 17, 64, 100, 521, 1000, 2000, 2790, 2800, 3000, 5000, 9000):
        N = rng.getrandbits(bits) | (1 << (bits - 1)) | 1
        Ns.append(N)
        Es.append(rng.getrandbits(rng.randint(1, 300)) | 1)
    Es[0] = 0xDEADBEEF
    for base in (2, 3, 53, 65535):
        got = mr.powm(Ns, Es, base)
        for N, E, r in zip(Ns, Es, got):
            assert r == pow(base, E, N) == _gmp_powm(base, E, N), (base, N.bit_length())


def test_powm_long_exponent(mr):
    rng = random.Random(7)
    N = rng.getrandbits(4000) | (1 << 3999) | 1
    E = rng.getrandbits(4000)
    assert mr.powm([N], [E], 2)[0] == pow(2, E, N)


def test_residue_equals_gmp_strong_residue(mr):
    rng = random.Random(11)
    Ns = [rng.getrandbits(b) | (1 << (b - 1)) | 1 for b in (200, 700, 1500, 2790, 2900, 6000)]
    for base in (2, 3):
        ver, res = mr.test(Ns, base)
        for N, v, r in zip(Ns, ver, res):
            s, rg = oracle.strong_residue(N, base)
            assert r == rg
            assert v == oracle.strong_test(N, base)


def test_mersenne_primes_all_witnesses(mr):
    Ms = [(1 << p) - 1 for p in (521, 607, 1279)]
    for a in WITNESSES:
        ver, _ = mr.test(Ms, a, residues=False)
        assert ver == [1, 1, 1], a


def test_nextprime_kats_s1_and_general_s(mr):
    base = 1 << 512
    primes = []
    p = base + 3
    while len(primes) < 3:  # s = 1 primes (p == 3 mod 4), correctness_tests.cuh:959-1031
        p = oracle.nextprime(p)
        if (p - 1) % 4 == 2:
            primes.append(p)
    for target in (2, 3, 4):  # s = 2, 3, >= 4
        p = base + 1
        while True:
            p = oracle.nextprime(p)
            s = ((p - 1) & -(p - 1)).bit_length() - 1
            if (target < 4 and s == target) or (target == 4 and s >= 4):
                primes.append(p)
                break
    for a in WITNESSES[:6]:
        ver, res = mr.test(primes, a)
        assert ver == [1] * len(primes), a
        for N, r in zip(primes, res):
            assert r == oracle.strong_residue(N, a)[1]


def test_random_composites_and_strong_pseudoprimes(mr):
    rng = random.Random(5)
    Ns = [rng.getrandbits(900) | (1 << 899) | 1 for _ in range(20)]
    Ns += [2047, 3277, 4033, 4681, 8321]  # base-2 strong pseudoprimes
    Ns += [3215031751, 25326001]           # pseudoprimes to several small bases
    for a in (2, 3, 5):
        ver, _ = mr.test(Ns, a, residues=False)
        assert ver == [oracle.strong_test(N, a) for N in Ns], a


def test_mixed_lengths_one_batch(mr):
    rng = random.Random(9)
    Ns = []
    for bits in (40, 2700, 2760, 5800, 11000, 23000, 45000, 90000, 150000, 166096, 200000, 332192):
        Ns.append(rng.getrandbits(bits) | (1 << (bits - 1)) | 1)
    Es = [rng.getrandbits(64) | 1 for _ in Ns]
    got = mr.powm(Ns, Es, 2)
    for N, E, r in zip(Ns, Es, got):
        assert r == pow(2, E, N), N.bit_length()


def test_invalid_inputs_flagged(mr):
    ver, _ = mr.test([10, 1, 7, 1 << 200, (1 << pfb200.MR_MAX_BITS + 1) + 1], 2, residues=False)
    assert ver == [-1, -1, 1, -1, -1]


def test_bucket_boundaries(mr):
    # largest modulus of each transform length, and one bit more
    rng = random.Random(13)
    Ns = []
    for lg in range(8, 16):
        rb = 22 * (1 << (lg - 1))
        for bits in (rb - 36, rb - 35):
            if bits <= pfb200.MR_MAX_BITS:
                Ns.append(rng.getrandbits(bits) | (1 << (bits - 1)) | 1)
    Es = [0xDEADBEEF for _ in Ns]
    got = mr.powm(Ns, Es, 2)
    for N, r in zip(Ns, got):
        assert r == pow(2, 0xDEADBEEF, N), N.bit_length()


def _golden(name):
    path = os.path.join(GOLD, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    return json.load(open(path))


def test_first16_survivors_full_size_residues(mr):
    """50 000-digit N and rev(N) of the first 16 sieve survivors: residues
    2^d mod N must hash to the GMP values and verdicts match the reference."""
    g = _golden("mr_50k_first16.json")
    recs = g["records"]
    Ns = [oracle.build_candidate(r["a"], r["b"], r["c"], r["k"], r["j"], bool(r["rev"])) for r in recs]
    ver, res = mr.test(Ns, 2)
    for r, N, v, x in zip(recs, Ns, ver, res):
        n16 = (N.bit_length() + 15) // 16
        assert hashlib.sha256(x.to_bytes(2 * n16, "little")).hexdigest() == r["sha256"], (r["k"], r["j"])
        assert v == r["sprp2"]
    if "ref_miller_rabin_test" in g:
        for i in range(0, len(recs), 2):
            k, j = recs[i]["k"], recs[i]["j"]
            want = g["ref_miller_rabin_test"]["%d,%d" % (k, j)]
            got = 0 if ver[i] == 0 else (2 if ver[i + 1] == 1 else 1)
            assert got == want


def test_resident_batch_stepwise_equals_one_shot(mr):
    """Advancing a resident batch in uneven chunks gives the one-shot result
    (state round-trips through device memory between launches)."""
    rng = random.Random(21)
    Ns = [rng.getrandbits(b) | (1 << (b - 1)) | 1 for b in (1200, 3000, 7000, 7001, 40000)]
    Ns.append((1 << 1279) - 1)
    want_v, want_r = mr.test(Ns, 3)
    b = pfb200.MRBatch(mr, Ns, 3)
    left = b.steps_left()
    assert left >= 40000
    done = 0
    for k in (1, 7, 500, 3000):
        b.advance(k)
        done += k
    assert b.pending() > 0
    v, _ = b.results()
    assert -2 in v  # unfinished candidates are reported, not guessed
    b.advance(left - done)
    assert b.pending() == 0
    v, r = b.results(residues=True)
    assert v == want_v and r == want_r
    b.close()


def _check_records(mr, recs):
    Ns = [oracle.build_candidate(r["a"], r["b"], r["c"], r["k"], r["j"], bool(r["rev"])) for r in recs]
    ver, res = mr.test(Ns, 2)
    for r, N, v, x in zip(recs, Ns, ver, res):
        n16 = (N.bit_length() + 15) // 16
        assert N.bit_length() == r["bits"]
        assert "%016x" % (x & (2**64 - 1)) == r["low64"], (r["a"], r["k"], r["j"], r["rev"])
        assert hashlib.sha256(x.to_bytes(2 * n16, "little")).hexdigest() == r["sha256"]
        assert v == r["sprp2"]


def test_uniform_batch_every_candidate_residue(mr):
    """Every number the 256-candidate 50 000-digit batch draws from (N and
    rev(N) of all 107 survivors): residues hash to GMP's, verdicts match."""
    g = _golden("mr_50k_survivors.json")
    assert len(g["records"]) == 214
    _check_records(mr, g["records"])


def test_uneven_batch_subset_residues(mr):
    """The first 128 of the 512 uneven-batch candidates (50 000 - 100 000
    digits; 12 of them at the shorter transform length, so both lengths share
    the batch's launches) against GMP: residues word for word (SHA-256 and
    low 64 bits), verdicts bit for bit."""
    from pfb200.workloads import uneven_tuples
    name = "mr_uneven_first128.json"
    if not os.path.exists(os.path.join(GOLD, name)):
        name = "mr_uneven_first32.json"
    recs = _golden(name)["records"]
    assert [(r["a"], r["b"], r["c"], r["k"], r["j"], bool(r["rev"])) for r in recs] == \
        uneven_tuples(512)[:len(recs)]
    assert len({r["bits"] > 22 * (1 << 13) - 36 for r in recs}) == 2  # both transform lengths
    _check_records(mr, recs)


def test_autotune_picks_a_timed_pair_and_results_hold(mr):
    """The autotuner times every (quantum, chunk) pair of a bucket and keeps
    the fastest; results after tuning are unchanged (the chunks replay as CUDA
    graphs with the tuned parameters)."""
    out = mr.autotune(12, 12)
    rows = [r for r in out["tried"] if r["logl"] == 12]
    assert len(rows) == 6 and all(r["squarings_per_s_1"] > 0 and r["squarings_per_s_2"] > 0 for r in rows)
    b1 = max(r["squarings_per_s_1"] for r in rows)
    b2 = max(r["squarings_per_s_2"] for r in rows)
    best = max(rows, key=lambda r: r["squarings_per_s_1"] / b1 + r["squarings_per_s_2"] / b2)
    assert out["chosen"][12] == (best["quantum"], best["chunk"])
    rng = random.Random(41)
    Ns = [rng.getrandbits(b) | (1 << (b - 1)) | 1 for b in (20000, 21000, 22000)]
    ver, res = mr.test(Ns, 2)
    for N, v, r in zip(Ns, ver, res):
        assert r == oracle.strong_residue(N, 2)[1] and v == oracle.strong_test(N, 2)


def test_small_moduli_long_s_and_bases_multiple_of_n(mr):
    """Tiny moduli, s up to 16 (Fermat primes), Mersenne primes with s = 1,
    and bases that are multiples of N, against GMP's strong test."""
    Ns = [3, 5, 7, 11, 13, 17, 257, 65537, 641 * 6700417, (1 << 61) - 1, (1 << 127) - 1, 2**64 + 13]
    for base in (2, 3, 7, 17, 257, 65535):
        ver, res = mr.test(Ns, base)
        for N, v, r in zip(Ns, ver, res):
            s, rg = oracle.strong_residue(N, base)
            assert r == rg, (N, base)
            assert v == oracle.strong_test(N, base), (N, base)
