"""The allocation-free sieve entry point against the regular one.

pfb_sieve_run_noalloc is for callers that cannot call cudaMalloc (device
memory reserved up front by another allocator, or loops that cannot take the
synchronisation of cudaFree).  It keeps its working memory in a fixed
__device__ array inside the library, so this test checks that two calls in a
row (the second reusing whatever the first left in that array) produce the
same masks, bit for bit, as pfb_sieve_run with its own allocations.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import pfb200
from conftest import primes_below

pytestmark = pytest.mark.gpu


def _noalloc():
    L = pfb200.lib()
    f = L.pfb_sieve_run_noalloc
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_longlong, C.c_longlong, C.c_longlong, C.c_int,
                  C.c_void_p, C.c_uint, C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def test_noalloc_matches_regular_entry_point_two_calls(torch):
    run = _noalloc()
    P = primes_below(3_000_000)
    d_primes = torch.from_numpy(P.view(np.int32)).cuda()
    # K = 9999 then 2500 (same small-prime limit, 10 000), then 700 (limit
    # 4096): the scratch goes from the longer small-prime lists to shorter
    # ones, so whatever a call leaves in it must not reach the next one
    cases = [((50000, 30000, 100), 9999), ((50001, 1098, 100), 2500), ((50002, 2095, 101), 700)]
    ref = pfb200.Sieve(P)
    for (a, b, c), K in cases:
        want = ref.run([(a, b, c)], K)
        d_mask = torch.full((pfb200.mask_bytes(K),), 0xAB, dtype=torch.uint8, device="cuda")
        rc = run(d_primes.data_ptr(), len(P), a, b, c, K, d_mask.data_ptr(), 0, None)
        assert rc == 0, pfb200.last_error()
        torch.cuda.synchronize()
        got = d_mask.cpu().numpy()
        assert (got == want).all(), (a, b, c, K)
        if K <= 2500:  # and against the oracle itself (restated trial_div_cpu)
            o = oracle.sieve_grid(P, a, b, c, K)
            assert (got[:len(o)] == o).all(), (a, b, c, K)
    ref.close()


def test_noalloc_repeated_entries(torch):
    """A list that repeats small primes more often than the fixed lists hold
    gives the mask of the list without repeats (each value is listed once)."""
    run = _noalloc()
    P = primes_below(300_000)
    noisy = np.concatenate([np.full(6000, 3, np.uint32), P[P < 10000], P, np.full(50, 7, np.uint32)])
    d_primes = torch.from_numpy(noisy.view(np.int32)).cuda()
    a, b, c, K = 50000, 30000, 100, 1200
    d_mask = torch.zeros(pfb200.mask_bytes(K), dtype=torch.uint8, device="cuda")
    assert run(d_primes.data_ptr(), len(noisy), a, b, c, K, d_mask.data_ptr(), 0, None) == 0
    torch.cuda.synchronize()
    o = oracle.sieve_grid(P, a, b, c, K)
    assert (d_mask.cpu().numpy()[:len(o)] == o).all()


def test_noalloc_or_in_and_limits(torch):
    run = _noalloc()
    P = primes_below(200_000)
    d_primes = torch.from_numpy(P.view(np.int32)).cuda()
    K = 100
    pre = np.zeros(313, dtype=np.uint32)
    pre[3] = 0xF0F0F0F0
    d_mask = torch.from_numpy(pre.view(np.int32).copy()).cuda()
    assert run(d_primes.data_ptr(), len(P), 15, 8, 3, K, d_mask.data_ptr(), pfb200.SIEVE_OR, None) == 0
    torch.cuda.synchronize()
    want = pfb200.trial_div_gpu(P, 15, 8, 3, pre.copy())
    assert (d_mask.cpu().numpy().view(np.uint32) == want).all()
    assert run(d_primes.data_ptr(), len(P), 15, 8, 3, 10000, d_mask.data_ptr(), 0, None) == pfb200.PFB_E_CAPACITY
