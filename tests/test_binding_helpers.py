"""The Python binding's own arithmetic, on the CPU: the candidates it builds
for the benches and tests (the reference formula, miller_rabin.c:32-74), the
16-bit limb conversions of pfb_mr_number_t and the mask unpacking."""
import random
import sys

import numpy as np

import oracle
import pfb200

sys.set_int_max_str_digits(0)


def test_build_candidate_equals_the_oracle():
    rng = random.Random(21)
    tuples = [(50000, 30000, 100, 1, 99), (100000, 60000, 100, 5, 84), (4, 2, 1, 3, 7), (12, 5, 2, 9999, 10)]
    for _ in range(60):
        a = rng.randint(20, 3000)
        c = rng.randint(0, a // 3)
        b = rng.randint(c + 5, a - 5)
        tuples.append((a, b, c, rng.randint(1, 9999), rng.randint(1, 9999)))
    for a, b, c, k, j in tuples:
        for rev in (False, True):
            if rev and (a - b - len(str(k)) < 0 or a - c - len(str(j)) < 0):
                continue
            assert pfb200.build_candidate(a, b, c, k, j, rev) == oracle.build_candidate(a, b, c, k, j, rev)


def test_limb_round_trip():
    rng = random.Random(22)
    for x in [0, 1, 65535, 65536, 2 ** 64 - 1] + [rng.getrandbits(b) for b in (17, 1000, 166097)]:
        limbs = pfb200.int_to_limbs16(x)
        assert limbs.dtype == np.uint16 and len(limbs) == max(1, (x.bit_length() + 15) // 16)
        assert pfb200.limbs16_to_int(limbs) == x
    st, keep = pfb200._numbers([12345, np.array([1, 2], dtype=np.uint16)])
    assert st[0].n_limbs == 1 and st[1].n_limbs == 2 and st[1].limbs[1] == 2 and len(keep) == 2


def test_unpack_mask_bit_order():
    K = 7
    mask = np.zeros(pfb200.mask_bytes(K), dtype=np.uint8)
    for k, j in [(1, 1), (1, 7), (3, 4), (7, 7)]:
        q = (k - 1) * K + (j - 1)  # bit q = (k-1) K + (j-1), LSB-first
        mask[q >> 3] |= 1 << (q & 7)
    m = pfb200.unpack_mask(mask, K)
    assert m.shape == (K, K) and m.sum() == 4
    assert m[0, 0] and m[0, 6] and m[2, 3] and m[6, 6]
