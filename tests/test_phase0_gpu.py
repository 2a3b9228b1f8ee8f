"""GPU Phase-0 table (pfb_phase0_*) against the reference's own Phase 0
(golden masks from sieve_table_build + sieve_apply) and the restatement."""
import json
import os

import numpy as np
import pytest

import oracle
import pfb200
import phase0

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "phase0_ref.json")


@pytest.fixture(scope="module")
def table():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    t = pfb200.Phase0(oracle.primes_below(10_000))
    yield t
    t.close()


def test_table_shape(table):
    info = table.info()
    assert info["primes"] == 62 and info["masks"] == 3_208_136
    assert info["table_bytes"] == 3_208_136 * 313 * 4


def test_masks_equal_reference(table):
    g = json.load(open(GOLD))
    abc = [tuple(c["abc"]) for c in g["cases"]]
    got = table.apply(abc)
    for case, m in zip(g["cases"], got):
        assert (m == np.frombuffer(bytes.fromhex(case["words_hex"]), dtype="<u4")).all(), case["abc"]


def test_random_triples_equal_restatement_and_or_semantics(table):
    rng = np.random.default_rng(17)
    abc = [(int(a), int(rng.integers(0, a)), int(rng.integers(0, 1000))) for a in rng.integers(1000, 200000, 6)]
    got = table.apply(abc)
    P = oracle.primes_below(10_000)
    for t, m in zip(abc, got):
        assert (m == phase0.phase0_mask(P, *t)).all(), t
    pre = rng.integers(0, 2**32, size=(len(abc), 313), dtype=np.uint32)
    assert (table.apply(abc, pre.copy(), or_in=True) == (pre | got)).all()


def test_phase0_premask_through_the_pipeline(table):
    """Phase-0 bits handed to the pipeline as its pre-mask (the reference's
    gpu_task_t.sieve_bits): the survivors are those of trial division with
    the Phase-0 bits OR-ed in."""
    P = oracle.primes_below(100_000)
    abc = [(60, 40, 20), (81, 61, 27)]
    pre = table.apply(abc)
    sv = pfb200.Sieve(P)
    mr = pfb200.MillerRabin(0)
    recs, st = pfb200.pipeline_run(sv, mr, abc, 100, pre_mask=pre.view(np.uint8).reshape(-1))
    want = []
    for t, (a, b, c) in enumerate(abc):
        m = oracle.sieve_grid(P, a, b, c, 100) | pre[t].view(np.uint8)[:1250]
        bits = np.unpackbits(m, bitorder="little")[:10000].reshape(100, 100)
        want += [(a, b, c, int(k) + 1, int(j) + 1) for k, j in zip(*np.nonzero(bits == 0))]
    assert [r[:5] for r in recs] == want
    sv.close()
    mr.close()
