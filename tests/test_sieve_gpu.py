"""GPU parity of the Phase-1 sieve against the reference and the oracle.

Mirrors the reference's tests/test_gpu.c (GPU vs CPU brute force, survivors
clean, determinism) through the drop-in ABI, and extends them to the wide
K x K grid against the restated trial_div_cpu (oracle/sieve_oracle.c).
Every comparison is bit-exact.
"""
import json
import os

import numpy as np
import pytest

import oracle
import pfb200
from conftest import primes_below

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _words(h):
    return np.frombuffer(bytes.fromhex(h), dtype="<u4").copy()


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_drop_in_reference_kat(torch_cuda):
    g = json.load(open(os.path.join(GOLD, "sieve_ref_kat.json")))
    p = np.array(g["primes"], dtype=np.uint32)
    for case in g["cases"]:
        a, b, c = case["abc"]
        bits = pfb200.trial_div_gpu(p, a, b, c)
        assert (bits == _words(case["words_hex"])).all(), case["abc"]


def test_drop_in_determinism_and_or_semantics(torch_cuda):
    p = primes_below(100)
    b1 = pfb200.trial_div_gpu(p, 15, 8, 3)
    b2 = pfb200.trial_div_gpu(p, 15, 8, 3)
    assert (b1 == b2).all()
    b3 = pfb200.trial_div_gpu(p, 25, 12, 6)
    b4 = pfb200.trial_div_gpu(p, 25, 12, 6)
    assert (b3 == b4).all()
    pre = np.zeros(313, dtype=np.uint32)
    pre[7] = 0xA5A5A5A5
    pre[312] = 0x0000FFFF
    out = pfb200.trial_div_gpu(p, 15, 8, 3, pre.copy())
    assert (out == (b1 | pre)).all()
    t = pfb200.GpuTiming()
    pfb200.trial_div_gpu(p, 15, 8, 3, None, t)
    assert t.kernel >= 0.0 and t.upload >= 0.0 and t.download >= 0.0


def test_drop_in_50000_30000_100_golden(torch_cuda, primes_1e8):
    g = json.load(open(os.path.join(GOLD, "sieve_50000_30000_100.json")))
    a, b, c = g["abc"]
    bits = pfb200.trial_div_gpu(primes_1e8, a, b, c)
    assert (bits == _words(g["words_hex"])).all()
    m = pfb200.unpack_mask(bits.view(np.uint8), 100)
    surv = [[k + 1, j + 1] for k in range(99) for j in range(99) if not m[k, j]]
    assert surv == g["survivors_99"] and len(surv) == 107


@pytest.mark.parametrize("K", [1, 7, 10, 99, 100, 101, 999, 1000, 1234])
def test_wide_grid_vs_oracle_small_primes(torch_cuda, K):
    rng = np.random.default_rng(1000 + K)
    P = primes_below(200_000)
    abc = []
    for _ in range(3):
        a = int(rng.integers(50, 3000))
        b = int(rng.integers(1, a))
        c = int(rng.integers(0, b))
        abc.append((a, b, c))
    abc.append((60, 57, 2))   # a-b-lk < 0 for lk >= 4
    abc.append((40, 20, 39))  # a-c-lj < 0 for lj >= 2
    masks = pfb200.trial_div_gpu_grid(P, abc, K)
    blk = pfb200.mask_bytes(K)
    for t, (a, b, c) in enumerate(abc):
        ref = oracle.sieve_grid(P, a, b, c, K)
        got = masks[t * blk: t * blk + len(ref)]
        assert (got == ref).all(), (K, a, b, c)
        assert not masks[t * blk + len(ref): (t + 1) * blk].any()


def test_wide_grid_k9999_vs_oracle(torch_cuda):
    # triples of the wide-grid enumeration (c from 100, b = c+1 + 997 i) with primes < 2e6
    P = primes_below(2_000_000)
    abc = [(50000, 101, 100), (50001, 101 + 997 * 7, 100), (50063, 101 + 997 * 40, 101)]
    s = pfb200.Sieve(P)
    masks = s.run(abc, 9999)
    blk = pfb200.mask_bytes(9999)
    for t, (a, b, c) in enumerate(abc):
        ref = oracle.sieve_grid(P, a, b, c, 9999)
        assert (masks[t * blk: t * blk + len(ref)] == ref).all(), (a, b, c)
    s.close()


def test_k9999_full_primes_subgrid_matches_reference(torch_cuda, primes_1e8):
    # (k,j) <= 100 of a K = 9999 run must equal the reference's 100 x 100 grid.
    g = json.load(open(os.path.join(GOLD, "sieve_50000_30000_100.json")))
    a, b, c = g["abc"]
    s = pfb200.Sieve(primes_1e8)
    m = pfb200.unpack_mask(s.run([(a, b, c)], 9999), 9999)
    ref = pfb200.unpack_mask(_words(g["words_hex"]).view(np.uint8), 100)
    assert (m[:100, :100] == ref).all()
    # survivors are clean and eliminations are justified on sampled pairs
    # (tests/test_gpu.c:95-139), by direct evaluation of N and rev(N) mod p
    P = primes_1e8.astype(np.uint64)
    r10 = {}

    def pw(e):
        if e not in r10:
            r10[e] = _powvec(10, e, P)
        return r10[e]

    rng = np.random.default_rng(7)
    for k, j in zip(rng.integers(1, 10000, size=40), rng.integers(1, 10000, size=40)):
        k, j = int(k), int(j)
        lk, lj = len(str(k)), len(str(j))
        rk, rj = int(str(k)[::-1]), int(str(j)[::-1])
        vN = (pw(a) + 3 * P - (k % P) * pw(b) % P - (j % P) * pw(c) % P - 1) % P
        eb, ec = a - b - lk, a - c - lj
        vR = (pw(a) + 3 * P - (rk % P) * pw(eb) % P - (rj % P) * pw(ec) % P - 1) % P
        hit = bool((vN == 0).any() or (vR == 0).any())
        assert m[k - 1, j - 1] == hit, (k, j)
    s.close()


def _powvec(base: int, e: int, P: np.ndarray) -> np.ndarray:
    """base^e mod p for every p in P (uint64, p < 2^31)."""
    r = np.ones_like(P)
    x = np.full_like(P, base) % P
    while e:
        if e & 1:
            r = r * x % P
        x = x * x % P
        e >>= 1
    return r


def test_multi_triple_equals_single(torch_cuda):
    P = primes_below(300_000)
    abc = [(5000, 3000, 100), (5001, 2000, 10), (6000, 5997, 5996)]
    s = pfb200.Sieve(P)
    many = s.run(abc, 500)
    blk = pfb200.mask_bytes(500)
    for t, tr in enumerate(abc):
        one = s.run([tr], 500)
        assert (many[t * blk:(t + 1) * blk] == one).all()
    s.close()


def test_device_mask_and_survivor_compaction(torch_cuda):
    torch = torch_cuda
    P = primes_below(1_000_000)
    K = 2500
    abc = [(50000, 30000, 100)]
    s = pfb200.Sieve(P)
    blk = pfb200.mask_bytes(K)
    d_mask = torch.zeros(blk, dtype=torch.uint8, device="cuda")
    s.run(abc, K, d_mask)
    torch.cuda.synchronize()
    host = s.run(abc, K)
    assert (d_mask.cpu().numpy() == host).all()
    m = pfb200.unpack_mask(host, K)
    expect = [(k + 1) << 16 | (j + 1) for k, j in zip(*np.nonzero(~m))]
    cap = len(expect) + 16
    d_out = torch.zeros(cap, dtype=torch.int32, device="cuda")
    n = s.survivors(d_mask, K, d_out, cap)
    assert n == len(expect)
    got = d_out[:n].cpu().numpy().view(np.uint32)
    assert (got == np.array(expect, dtype=np.uint32)).all()
    # too small a buffer reports the count and PFB_E_CAPACITY without overflow
    small = torch.zeros(8, dtype=torch.int32, device="cuda")
    assert s.survivors(d_mask, K, small, 8) == len(expect)
    s.close()


def test_k_changes_on_one_caller_stream(torch_cuda):
    """Asynchronous calls on a caller's stream with K changing between them:
    a call whose K needs a new split of the prime list first waits for the
    stream's earlier calls, so every mask equals the oracle's."""
    torch = torch_cuda
    P = primes_below(100_000)
    s = pfb200.Sieve(P)
    stream = torch.cuda.Stream()
    abc = (81, 61, 27)
    Ks = [3000, 100, 3000, 40, 1200]  # small-prime limits 10^4, 4096, 10^4, 4096, 10^4
    masks = [torch.zeros(pfb200.mask_bytes(K), dtype=torch.uint8, device="cuda") for K in Ks]
    for K, m in zip(Ks, masks):
        s.run([abc], K, m, stream=stream.cuda_stream)
    stream.synchronize()
    for K, m in zip(Ks, masks):
        want = oracle.sieve_grid(P, *abc, K)
        assert (m.cpu().numpy()[:len(want)] == want).all(), K
    s.close()


def test_bad_arguments_rejected(torch_cuda):
    P = primes_below(1000)
    with pytest.raises(pfb200.PfbError):
        pfb200.trial_div_gpu_grid(P, [(10, 5, 1)], 10000)
    with pytest.raises(pfb200.PfbError):
        pfb200.trial_div_gpu_grid(P, [(10, -5, 1)], 100)


def test_drop_in_equals_reference_gpu_kernel(torch_cuda, primes_1e8):
    """The reference's own trial_div_gpu (trial_div.cu, built unmodified for
    sm_100a) and the drop-in give the same 313 words: the test_gpu.c triples
    with its primes 3..97 (tests/test_gpu.c:158-177), OR-in on a pre-set
    mask, and (50000, 30000, 100) with every odd prime below 1e8."""
    if not oracle.ref_gpu_available():
        pytest.skip("reference GPU sieve not built (oracle/_ref)")
    small = primes_below(97)
    pre = np.zeros(313, dtype=np.uint32)
    pre[[0, 100, 312]] = [0x1, 0xF0F0F0F0, 0x80]
    for (a, b, c), P, start in [((15, 8, 3), small, None), ((20, 10, 5), small, None),
                                ((25, 12, 6), small, pre), ((50000, 30000, 100), primes_1e8, None)]:
        want, rc, _ = oracle.ref_trial_div_gpu(P, a, b, c, None if start is None else start.copy())
        assert rc == 0
        got = pfb200.trial_div_gpu(P, a, b, c, None if start is None else start.copy())
        assert (got == want).all(), (a, b, c)


def test_k9999_full_grid_all_primes_vs_oracle_hashes(torch_cuda, primes_1e8):
    """The wide-grid workload at full size: K = 9999 (99 980 001 pairs) with
    every odd prime below 1e8, four triples in one call.  Each mask must hash
    to the oracle's (restated trial_div_cpu; tests/golden/sieve_k9999_full.json,
    made by tests/golden/make_sieve_k9999_golden.py), with the same number of
    survivors and the same first survivors in k-major order."""
    import hashlib
    path = os.path.join(GOLD, "sieve_k9999_full.json")
    if not os.path.exists(path):
        pytest.skip("sieve_k9999_full.json not generated")
    g = json.load(open(path))
    K = g["K"]
    assert K == 9999 and g["primes"] == len(primes_1e8)
    abc = [tuple(r["abc"]) for r in g["records"]]
    s = pfb200.Sieve(primes_1e8)
    masks = s.run(abc, K)
    blk, nb = pfb200.mask_bytes(K), g["mask_bytes"]
    for t, r in enumerate(g["records"]):
        m = masks[t * blk: t * blk + nb]
        assert hashlib.sha256(m.tobytes()).hexdigest() == r["sha256"], r["abc"]
        bits = np.unpackbits(m, bitorder="little")[:K * K]
        assert K * K - int(bits.sum()) == r["survivors"]
        idx = np.flatnonzero(bits == 0)[:len(r["first_survivors"])]
        assert [[int(q // K) + 1, int(q % K) + 1] for q in idx] == r["first_survivors"]
    s.close()
