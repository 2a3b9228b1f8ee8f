"""bench.py's bookkeeping on the CPU: the reference-structure work count the
roofline divides by, and the small kernel cases used for ncu captures."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_work_count():
    """M(L) = 2 (6 (L/2) log2 L + 3 L) modmuls x 3 INT32 multiplies per
    squaring: 9.44 M at 50 000 digits (L = 2^15 in the reference's 16-bit
    limbs, ntt_merge.cuh:21-24) and 20.05 M at 100 000 digits (L = 2^16)."""
    assert bench.ref_modmuls_per_squaring(50000) * bench.SQ_PER_MODMUL == 9437184
    assert bench.ref_modmuls_per_squaring(100000) * bench.SQ_PER_MODMUL == 20054016
    L = 1 << 15
    assert bench.ref_modmuls_per_squaring(50000) == 2 * (6 * (L // 2) * 15 + 3 * L)


def test_mr_cases_are_eight_candidates():
    for name, (abc, pairs) in bench.MR_CASES.items():
        a, b, c = abc
        assert c < b < a
        if pairs is not None:
            assert len(pairs) == 4  # N and rev(N) of each: 8 candidates, one CTA each


def test_sieve_input_primes():
    P = bench.odd_primes_below(1_000_000)
    assert len(P) == 78497 and P[0] == 3 and P[-1] == 999983  # pi(10^6) = 78498, less the prime 2
    assert len(bench.odd_primes_below(100)) == 24


def test_e2e_breakdown_stages_with_a_stand_in_batch():
    """bench.e2e_breakdown's control flow (the stages of one test call through
    the batch API) on a stand-in batch object: main advance by the steps left,
    top-up rounds until nothing is pending, then the read-back."""
    class Batch:
        def __init__(self, eng, cands, base):
            self.left, self.pend, self.done, self.closed = 1000, 3, 0, False

        def steps_left(self):
            return self.left

        def advance(self, steps):
            self.done += steps
            self.left = max(0, self.left - steps)
            if steps == 4096:
                self.pend = max(0, self.pend - 1)

        def pending(self):
            return self.pend

        def results(self, residues=False):
            return [0], [0]

        def close(self):
            self.closed = True

    class Fake:
        MRBatch = Batch

        @staticmethod
        def batch_steps_done(b):
            return b.done

    class Torch:
        class cuda:
            @staticmethod
            def synchronize():
                pass

    out = bench.e2e_breakdown(Fake, Torch, None, [1, 2])
    assert out["topup_rounds"] == 3 and out["steps_main"] == 1000 and out["steps_topup"] == 3 * 4096
    assert all(out[k] >= 0 for k in ("setup_s", "main_s", "topup_s", "results_s"))


def test_reference_arm_line():
    """bench.py --impl reference (the reference's CPU path, timed on the host
    cores) prints one JSON line with the contract's keys; under a launcher,
    ranks other than 0 print nothing and exit 0."""
    import json
    import os
    import subprocess
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
           "--no-calibration"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == "tests/s"
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"] and line["higher_is_better"] is True
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["cores"] >= 1
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r1 = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r1.returncode == 0 and r1.stdout.strip() == ""
