"""Continuous batching: results are the same alone and in the mix.

Candidates of different lengths are streamed into the server while others
are resident (staggered submission), and each verdict and residue must equal
the one-candidate-per-call result and GMP's (oracle), word for word.
"""
import hashlib
import json
import os
import random
import time

import pytest

import oracle
import pfb200

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    e = pfb200.MillerRabin(0)
    yield e
    e.close()


def _numbers(seed, n):
    rng = random.Random(seed)
    out = []
    for i in range(n):
        bits = rng.choice([700, 1500, 3000, 2790, 6000, 9000, 12000])
        out.append(rng.getrandbits(bits) | (1 << (bits - 1)) | 1)
    out[3] = (1 << 1279) - 1          # a prime (passes)
    out[5] = oracle.nextprime(1 << 700)
    return out


def _drain(srv, want, timeout_s=120):
    got = {}
    t0 = time.time()
    while len(got) < want and time.time() - t0 < timeout_s:
        for r in srv.poll(64, 200):
            got[r["tag"]] = r
    return got


def test_alone_equals_in_the_mix(engine):
    Ns = _numbers(1, 24)
    alone = [engine.test([N], 2) for N in Ns]          # one candidate per call
    srv = pfb200.MRServer(engine, max_resident=6, chunk_steps=256)
    got = {}
    for i, N in enumerate(Ns):                       # arrivals while others run
        srv.submit(N, tag=i, residue=True)
        if i % 5 == 4:
            time.sleep(0.05)
            for r in srv.poll(64, 10):
                got[r["tag"]] = r
    got.update(_drain(srv, len(Ns) - len(got)))
    st = srv.stats()
    srv.close()
    assert len(got) == len(Ns), st
    for i, N in enumerate(Ns):
        v_alone, r_alone = alone[i][0][0], alone[i][1][0]
        assert got[i]["verdict"] == v_alone == oracle.strong_test(N, 2)
        assert got[i]["residue"] == r_alone == oracle.strong_residue(N, 2)[1]
        assert got[i]["submit_s"] <= got[i]["admit_s"] <= got[i]["done_s"]
    assert st["launches"] > 1 and st["completed"] == len(Ns)


def test_budget_limits_admission(engine):
    Ns = _numbers(2, 8)
    srv = pfb200.MRServer(engine, max_resident=8, hbm_budget_bytes=150_000, chunk_steps=128)
    for i, N in enumerate(Ns):
        srv.submit(N, tag=i, residue=True)
    got = _drain(srv, len(Ns))
    st = srv.stats()
    srv.close()
    assert st["bytes_owned"] <= 150_000 and st["completed"] == len(Ns)
    for i, N in enumerate(Ns):
        assert got[i]["residue"] == oracle.strong_residue(N, 2)[1]


def test_invalid_requests_reported(engine):
    srv = pfb200.MRServer(engine, max_resident=2)
    srv.submit(10, tag=1)
    srv.submit(1 << 400, tag=2)
    srv.submit(2047, tag=3)   # base-2 strong pseudoprime
    got = _drain(srv, 3, 60)
    srv.close()
    assert got[1]["verdict"] == -1 and got[2]["verdict"] == -1 and got[3]["verdict"] == 1


def test_full_size_requests_in_the_mix(engine):
    """Ten 50 000 - 100 000-digit requests of the uneven workload (both
    transform lengths: four at <= 54 250 digits) through a server with eight
    slots: two requests wait for a slot and are admitted while the others run.
    Every residue must hash to GMP's (tests/golden/mr_uneven_first32.json)."""
    path = os.path.join(os.path.dirname(__file__), "golden", "mr_uneven_first32.json")
    recs = json.load(open(path))["records"]
    pick = [0, 1, 2, 4, 6, 3, 5, 7, 22, 23]   # 3, 5, 22, 23: the shorter transform length
    assert sum(1 for i in pick if recs[i]["a"] <= 54250) == 4
    srv = pfb200.MRServer(engine, max_resident=8, chunk_steps=256)
    Ns = {}
    for i in pick:
        r = recs[i]
        Ns[i] = oracle.build_candidate(r["a"], r["b"], r["c"], r["k"], r["j"], bool(r["rev"]))
        srv.submit(Ns[i], tag=i, residue=True)
    got = _drain(srv, len(pick), timeout_s=600)
    st = srv.stats()
    srv.close()
    assert len(got) == len(pick), st
    assert max(g["admit_s"] for g in got.values()) > min(g["done_s"] for g in got.values())  # admitted mid-run
    for i in pick:
        r, N, x = recs[i], Ns[i], got[i]["residue"]
        n16 = (N.bit_length() + 15) // 16
        assert "%016x" % (x & (2**64 - 1)) == r["low64"], i
        assert hashlib.sha256(x.to_bytes(2 * n16, "little")).hexdigest() == r["sha256"], i
        assert got[i]["verdict"] == r["sprp2"]


def test_slot_allocation_failure_recovery(engine):
    """The server's recovery when slot memory cannot be allocated, driven by
    host-side fault injection (pfb_mr_server_inject_alloc_failures; the
    device never faults): with nothing resident, a request whose allocation
    and retry both fail is reported with verdict -1; with candidates
    resident, it is requeued and admitted once memory comes back, and its
    residue still equals GMP's."""
    rng = random.Random(17)
    srv = pfb200.MRServer(engine, max_resident=8, chunk_steps=256)
    assert srv.inject_alloc_failures(2) == 0
    srv.submit(rng.getrandbits(3000) | 1 | (1 << 2999), tag=0, residue=True)
    got = _drain(srv, 1, 60)
    assert got[0]["verdict"] == -1
    assert srv.inject_alloc_failures(0) == 2
    # two long requests become resident; then three allocations fail
    longs = [rng.getrandbits(60000) | 1 | (1 << 59999) for _ in range(2)]
    for i, N in enumerate(longs):
        srv.submit(N, tag=10 + i, residue=True)
    t0 = time.time()
    while srv.stats()["resident"] < 2 and time.time() - t0 < 60:
        time.sleep(0.01)
    assert srv.stats()["resident"] == 2
    srv.inject_alloc_failures(3)
    shorts = [rng.getrandbits(b) | 1 | (1 << (b - 1)) for b in (2000, 5000, 9000)]
    for i, N in enumerate(shorts):
        srv.submit(N, tag=20 + i, residue=True)
    got = _drain(srv, 5, 300)
    used = srv.inject_alloc_failures(0)
    srv.close()
    assert used == 5 and len(got) == 5
    for tag, N in list(zip((10, 11), longs)) + list(zip((20, 21, 22), shorts)):
        assert got[tag]["verdict"] == oracle.strong_test(N, 2)
        assert got[tag]["residue"] == oracle.strong_residue(N, 2)[1]
