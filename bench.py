#!/usr/bin/env python
"""Benchmark of the two hot paths on B200.

Headline (value): base-2 strong probable-prime tests per second of the
served, batched Miller-Rabin engine on the uniform 50 000-digit batch: 256
candidates, N and rev(N) for 128 (k,j) drawn with splitmix64(seed=1) from the
sieve survivors (k,j <= 99) of (a,b,c) = (50000, 30000, 100).  The survivors
come from this repository's own GPU sieve over every odd prime below 1e8.

A step is `--chunk` modular squarings of every candidate of the resident
batch; tests/s = candidates * squarings done / squarings per test / time.
Beside it the line reports:
  e2e          complete tests through the C ABI (pfb_mr_test) from host limbs:
               host set-up, H2D, every squaring, verdict + residue D2H
  plain        the one-candidate-per-call form on the same GPU
  sieve        K = 9999 grid pairs/s over the (a,b,c) triples of the
               wide-grid triple enumeration, and the drop-in 100 x 100 call
  roofline     INT32 multiplies of the reference's squaring structure
               (6 length-L transforms + 3 pointwise products, 2 primes, 3
               multiplies per modmul, L = 32768 at 50 000 digits) per second,
               over this device's measured INT32 multiply peak
  cpu_baseline GMP 6.3 mpz_powm on the host cores, sampled

Multi-GPU: one process per GPU (torchrun), each an independent replica
(weak scaling); the time is the max over ranks.
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "prime-finder_b200"))
sys.set_int_max_str_digits(0)
from pfb200 import replicas  # noqa: E402
from pfb200.workloads import serving_draw, sieve_triples, uneven_tuples, uniform_batch_pairs  # noqa: E402

SQ_PER_MODMUL = 3  # INT32 multiplies per modular multiplication (reference count)
METRIC = "MR base-2 tests/s, uniform batch of 256 x 50 000-digit candidates, served/batched"
WORKLOAD = ("uniform MR batch: 256 x 50 000-digit N/rev(N), (k,j) from the (50000,30000,100) sieve "
            "survivors, splitmix64 seed 1")
# dram__bytes_read.sum + dram__bytes_write.sum of the timed persist_kernel launch of
# the uniform batch (1024 squarings x 256 candidates, L2 flushed before it), from one
# ncu capture of this build (profiles/persist_kernel_uniform_batch_dram.txt), in a run
# whose autotuner chose 16-step quanta at L = 2^14: a run with longer quanta re-reads
# the residues less often
PERSIST_LAUNCH_DRAM_BYTES = 73122560 + 30478080
PERSIST_LAUNCH_DRAM_QUANTUM = 16


def ref_modmuls_per_squaring(digits: int) -> int:
    """Modmuls of one squaring in the reference's structure (16-bit limbs,
    limbs_for_digits + padding to a power of two, 6 transforms, 3 pointwise
    products, 2 word primes): M(L) = 2 (6 (L/2) log2 L + 3 L)."""
    limbs = int((digits * 3.32193 + 15) / 16) + 4
    L = 1
    while L < 2 * limbs:
        L *= 2
    lg = L.bit_length() - 1
    return 2 * (6 * (L // 2) * lg + 3 * L)


# --------------------------------------------------------------- clocks ----

class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------- CPU baseline ---

def _gmp_powm_sample(args):
    a, b, c, k, j, rev, sample_bits = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    N = oracle.build_candidate(a, b, c, k, j, rev)
    d = (N - 1) >> 1
    E = d >> max(0, d.bit_length() - sample_bits)
    n16 = (N.bit_length() + 15) // 16
    nl = oracle.int_to_limbs(N, n16)
    el = oracle.int_to_limbs(E, (E.bit_length() + 15) // 16)
    bl = oracle.int_to_limbs(2, 1)
    out = np.zeros(n16, dtype=np.uint16)
    L = oracle.lib()
    t0 = time.perf_counter()
    L.oracle_powm(oracle._ptr(bl, oracle.C.c_uint16), 1, oracle._ptr(el, oracle.C.c_uint16), len(el),
                  oracle._ptr(nl, oracle.C.c_uint16), n16, oracle._ptr(out, oracle.C.c_uint16))
    dt = time.perf_counter() - t0
    return dt / E.bit_length(), d.bit_length()


def _reference_full_test(abc, kj, q):
    """One call of the reference's own miller_rabin_test (oracle/_ref, built
    from miller_rabin.c) on N(a,b,c,k,j), timed on one core."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_available():
        return
    t0 = time.perf_counter()
    code = oracle.ref_miller_rabin_test(abc[0], abc[1], abc[2], kj[0], kj[1])
    q.put({"full_test_s": time.perf_counter() - t0, "miller_rabin_test": code,
           "what": "reference miller_rabin_test(%d, %d, %d, %d, %d): GMP mpz_probab_prime_p(N, 5) on a "
                   "composite 50 000-digit N, one core" % (abc[0], abc[1], abc[2], kj[0], kj[1])})


def cpu_mr_baseline(pairs, abc, sample_bits=4096, procs=None):
    """GMP mpz_powm(2, d, N) on every host core at once, each on the top
    `sample_bits` bits of d; scaled to full tests (bits(d) squarings)."""
    procs = procs or os.cpu_count() or 1
    jobs = [(abc[0], abc[1], abc[2], pairs[i % len(pairs)][0], pairs[i % len(pairs)][1], bool(i & 1),
             sample_bits) for i in range(procs)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_gmp_powm_sample, jobs)
    wall = time.perf_counter() - t0
    per_core = [1.0 / (t_sq * bits) for t_sq, bits in res]
    return {"value": sum(per_core), "unit": "tests/s", "cores": procs, "kind": "port",
            "per_core": statistics.mean(per_core),
            "sample": "GMP 6.3 mpz_powm(2, top %d bits of d, N) for N, rev(N) of the 50 000-digit "
                      "batch, one process per core, scaled to bits(d) squarings per test (%.1f s wall)"
                      % (sample_bits, wall)}


def _sieve_ref_sample(args):
    stride, a, b, c = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    P = oracle.primes_below(100_000_000)
    sub = P[::stride].copy()
    t0 = time.perf_counter()
    oracle.ref_trial_div_cpu(sub, a, b, c)
    return (time.perf_counter() - t0) / len(sub), len(P)


def cpu_sieve_baseline(procs=None, stride_ref=20, stride_k9999=100):
    """Two CPU sieve baselines, both in pairs/s:
    value: the restated trial_div_cpu (oracle/sieve_oracle.c, OpenMP over the
      primes) on the K = 9999 grid of the GPU's workload, on every host core,
      over every 100th prime below 1e8, scaled by prime count;
    reference_100x100: the reference's own trial_div_cpu (its fixed 100 x 100
      grid) on every core, one process per core as the reference's CPU ranks
      run it, each over every 20th prime, scaled by prime count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    procs = procs or os.cpu_count() or 1
    P = oracle.primes_below(100_000_000)
    sub = P[::stride_k9999].copy()
    t0 = time.perf_counter()
    oracle.sieve_grid(sub, 50000, 30000, 100, 9999, threads=procs)
    t_k = (time.perf_counter() - t0) * len(P) / len(sub)
    out = {"value": 9999 * 9999 / t_k, "unit": "pairs/s", "cores": procs, "kind": "port",
           "sample": "restated trial_div_cpu (oracle/sieve_oracle.c) on the K = 9999 grid of (50000, 30000, "
                     "100), every %d-th prime < 1e8 on %d threads (%.1f s wall), scaled by prime count"
                     % (stride_k9999, procs, t_k * len(sub) / len(P))}
    if oracle.ref_available():
        ctx = mp.get_context("spawn")
        with ctx.Pool(procs) as pool:
            res = pool.map(_sieve_ref_sample, [(stride_ref, 50000 + i, 30000, 100) for i in range(procs)])
        per_core = [1e4 / (t_p * n) for t_p, n in res]
        out["reference_100x100"] = {
            "value": sum(per_core), "unit": "pairs/s", "cores": procs, "kind": "reference",
            "sample": "reference trial_div_cpu (its 100x100 grid) over every %d-th prime < 1e8, one process "
                      "per core, scaled by prime count" % stride_ref}
    return out


def reference_gpu_sieve(primes, abc, ours_words):
    """The reference's own trial_div_gpu (trial_div.cu, built unmodified for
    sm_100a into oracle/_ref) on the same triple and prime list as the
    drop-in: one untimed call, then two timed by its own gpu_timing_t; its 313
    words must equal the drop-in's."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_gpu_available():
        return None
    bits, rc, _ = oracle.ref_trial_div_gpu(primes, *abc)
    if rc != 0:
        return {"error": "trial_div_gpu returned %d" % rc}
    calls = []
    for _ in range(2):
        t0 = time.perf_counter()
        bits, rc, tm = oracle.ref_trial_div_gpu(primes, *abc)
        tm["call_s"] = time.perf_counter() - t0
        calls.append(tm)
    return {"kind": "reference", "build": "reference trial_div.cu, nvcc -O3 --use_fast_math, sm_100a",
            "call_s": statistics.mean(c["call_s"] for c in calls),
            "kernel_s": statistics.mean(c["kernel"] for c in calls),
            "upload_s": statistics.mean(c["upload"] for c in calls),
            "same_words": bool((bits == ours_words).all())}


def e2e_breakdown(pfb200, torch, eng, cands):
    """The stages of one pfb_mr_test call, timed apart through the batch API
    (the same calls run_jobs makes): host set-up + uploads + set-up kernel,
    the main advance by the longest test's steps, the rounds that finish the
    candidates the round-robin left behind, and the read-back."""
    t0 = time.perf_counter()
    b = pfb200.MRBatch(eng, cands, 2)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    b.advance(b.steps_left())
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    done_main = pfb200.batch_steps_done(b)
    rounds = 0
    while b.pending() and rounds < 1000:
        b.advance(4096)
        rounds += 1
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    done_all = pfb200.batch_steps_done(b)
    b.results(residues=True)
    t4 = time.perf_counter()
    b.close()
    return {"setup_s": t1 - t0, "main_s": t2 - t1, "topup_s": t3 - t2, "topup_rounds": rounds,
            "results_s": t4 - t3, "steps_main": done_main, "steps_topup": done_all - done_main}


def odd_primes_below(lim):
    """Odd primes <= lim by a plain Eratosthenes in numpy (the sieve's input data)."""
    import numpy as np
    sieve = np.ones(lim // 2 + 1, dtype=bool)
    sieve[0] = False
    for i in range(1, int(lim ** 0.5) // 2 + 1):
        if sieve[i]:
            p = 2 * i + 1
            sieve[p * p // 2::p] = False
    primes = (2 * np.nonzero(sieve)[0] + 1).astype(np.uint32)
    return primes[primes <= lim]


def sieve_case():
    """One triple, (50000, 30000, 100), on the 9999 x 9999 grid with every odd
    prime below 1e8 (the case of the sieve's ncu captures): one untimed call,
    then one timed with CUDA events."""
    import torch
    import pfb200
    sv = pfb200.Sieve(odd_primes_below(100_000_000), 0)
    stream = torch.cuda.Stream()
    dmask = torch.zeros(pfb200.mask_bytes(9999), dtype=torch.uint8, device="cuda")
    sv.run([(50000, 30000, 100)], 9999, dmask, stream=stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sv.run([(50000, 30000, 100)], 9999, dmask, stream=stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    print(json.dumps({"case": "sieve K=9999 (50000, 30000, 100), primes < 1e8", "ms": e0.elapsed_time(e1)}))
    sv.close()


def radix_case(ctas=592, reps=20):
    """The first radix-16 pass of a 2^14-point transform (both primes, 592
    CTAs = 4 per SM of work, each on its own random limbs) as the engine's
    butterfly pass and as an exact int8 byte-plane product on the tensor
    cores; the two forms' outputs must agree word for word."""
    import pfb200
    eng = pfb200.MillerRabin(0)
    r = pfb200.radix16_forms(eng, ctas, reps)
    eng.close()
    n = 1 << 14
    r.update({"case": "radix-16 pass, 2^14 points, 2 primes", "ctas": ctas,
              "points_per_s_butterfly": ctas * 2 * n / (r["ms_butterfly"] / 1e3),
              "points_per_s_tensor": ctas * 2 * n / (r["ms_tensor"] / 1e3) if r["ms_tensor"] > 0 else None})
    print(json.dumps(r))


# small cases of the squaring kernel for ncu captures: N and rev(N) of four
# (k, j) at one (a, b, c), 8 candidates (one CTA each), one launch of 64 squarings
MR_CASES = {
    "50k": ((50000, 30000, 100), None),  # the first four survivors of (50000, 30000, 100)
    "100k": ((100000, 60000, 100), [(1, 99), (2, 84), (4, 60), (5, 84)]),
}


def mr_case(name):
    """Run one small case of the persistent squaring kernel and print its time."""
    import torch
    import pfb200
    abc, pairs = MR_CASES[name]
    if pairs is None:
        g = json.load(open(os.path.join(ROOT, "tests", "golden", "sieve_50000_30000_100.json")))
        pairs = [tuple(x) for x in g["survivors_99"][:4]]
    cands = [pfb200.build_candidate(*abc, k, j, rev) for (k, j) in pairs for rev in (False, True)]
    eng = pfb200.MillerRabin(0)
    batch = pfb200.MRBatch(eng, cands, 2)
    stream = torch.cuda.Stream()
    batch.advance(64, stream.cuda_stream)  # the launch an ncu capture with -c 1 sees
    stream.synchronize()
    ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.advance(64, stream.cuda_stream)
        e1.record(stream)
        stream.synchronize()
        ms.append(e0.elapsed_time(e1))
    print(json.dumps({"case": name, "candidates": len(cands), "squarings_per_launch": 64,
                      "ms_per_launch": statistics.mean(ms), "us_per_squaring": 1e3 * statistics.mean(ms) / 64,
                      "steps_done": pfb200.batch_steps_done(batch)}))
    batch.close()
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--chunk", type=int, default=1024, help="squarings per candidate per step")
    ap.add_argument("--e2e-batch", type=int, default=0, help="candidates in the e2e call (0 = the whole batch)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-calibration", action="store_true",
                    help="reference arm: skip the full-length miller_rabin_test timed beside the samples")
    ap.add_argument("--no-uneven", action="store_true", help="skip the 512-candidate uneven batch")
    ap.add_argument("--sieve-triples", type=int, default=4)
    ap.add_argument("--serve-secs", type=float, default=None,
                    help="seconds of Poisson arrivals of 50k-100k-digit requests for the serving leg, which "
                         "then drains (default 180 on one GPU, 0 = no serving leg; off under torchrun)")
    ap.add_argument("--serve-drain", type=float, default=480.0,
                    help="longest wait for the requests in flight once arrivals stop")
    ap.add_argument("--serve-load", type=float, default=1.2, help="arrival rate / measured capacity")
    ap.add_argument("--mr-case", choices=sorted(MR_CASES) + ["all"],
                    help="only run a small case of the squaring kernel (8 candidates, 64 squarings; for ncu)")
    ap.add_argument("--e2e-breakdown", action="store_true",
                    help="also time the stages of the e2e call apart (one more e2e-sized run)")
    ap.add_argument("--sieve-case", action="store_true",
                    help="only run one K = 9999 sieve triple twice (for ncu)")
    ap.add_argument("--radix-case", action="store_true",
                    help="only time one radix-16 transform pass in its butterfly and tensor-core forms")
    args = ap.parse_args()
    if args.radix_case:
        radix_case()
        return
    if args.sieve_case:
        sieve_case()
        return
    if args.mr_case:
        for name in (sorted(MR_CASES) if args.mr_case == "all" else [args.mr_case]):
            mr_case(name)
        return

    rank, world, local = replicas.rank_world()
    abc1 = (50000, 30000, 100)

    if args.impl == "reference":
        if rank != 0:
            return
        import json as _j
        g = _j.load(open(os.path.join(ROOT, "tests", "golden", "sieve_50000_30000_100.json")))
        pairs = [tuple(x) for x in g["survivors_99"]]
        batch_pairs = uniform_batch_pairs(pairs)
        cores = os.cpu_count() or 1
        # calibration: the reference's own miller_rabin_test (GMP BPSW on N; N is
        # composite, so one full 50 000-digit base-2 powm) on one core, beside the samples
        ctx = mp.get_context("spawn")
        cal_q = ctx.Queue()
        cal = ctx.Process(target=_reference_full_test, args=(abc1, batch_pairs[0], cal_q))
        if not args.no_calibration:
            cal.start()
        t0 = time.perf_counter()
        steps = []
        for _ in range(args.warmup + args.steps):
            steps.append(cpu_mr_baseline(batch_pairs, abc1, sample_bits=1024, procs=max(1, cores - 1)))
        per_core = statistics.mean(s["per_core"] for s in steps[args.warmup:])
        v = per_core * cores
        calib = None
        if not args.no_calibration:
            try:
                calib = cal_q.get(timeout=900)
                est = 1.0 / statistics.mean(s["per_core"] for s in steps)
                calib["sampled_estimate_s"] = est
                calib["estimate_over_full"] = est / calib["full_test_s"]
            except Exception:
                pass
            cal.join(timeout=10)
            if cal.is_alive():
                cal.terminate()
        last = steps[-1]
        print(json.dumps({
            "impl": "reference", "metric": METRIC,
            "value": v, "unit": "tests/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * (time.perf_counter() - t0) / max(1, len(steps)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "candidates": 256, "parallelism": "replicas"},
            "cpu_baseline": {"kind": last["kind"], "cores": cores,
                             "sample": last["sample"] + "; per-core rate x %d cores" % cores, "value": v,
                             "unit": "tests/s", "calibration": calib},
            "e2e": {"value": v, "unit": "tests/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    # CPU baselines first: spawn pools before CUDA is initialised in this process
    cpu = None
    cpu_sieve = None
    if rank == 0 and not args.no_cpu:
        import json as _j
        g = _j.load(open(os.path.join(ROOT, "tests", "golden", "sieve_50000_30000_100.json")))
        pairs = [tuple(x) for x in g["survivors_99"]]
        cpu = cpu_mr_baseline(uniform_batch_pairs(pairs), abc1, sample_bits=4096)
        cpu_sieve = cpu_sieve_baseline()

    import numpy as np
    import torch
    import pfb200

    torch.cuda.set_device(local)
    dev = local
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, "cuda")

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    primes = odd_primes_below(100_000_000)

    # --- sieve -------------------------------------------------------------
    sv = pfb200.Sieve(primes, dev)
    m100 = sv.run([abc1], 100)
    ok = pfb200.unpack_mask(m100, 100)
    survivors = [(k + 1, j + 1) for k in range(99) for j in range(99) if not ok[k, j]]
    K = 9999
    stream = torch.cuda.Stream()
    blk = pfb200.mask_bytes(K)
    ntr = args.sieve_triples
    dmask = torch.zeros(blk * ntr, dtype=torch.uint8, device="cuda")
    sieve_launches = 0
    with torch.cuda.stream(stream):
        # every rank sieves its own shard of the triple enumeration (weak scaling)
        triples = replicas.shard(sieve_triples(ntr * (args.steps + args.warmup) * world), rank, world)
        for w in range(args.warmup):
            sv.run(triples[w * ntr:(w + 1) * ntr], K, dmask, stream=stream.cuda_stream)
        stream.synchronize()
        times = []
        for s in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            tr = triples[(args.warmup + s) * ntr:(args.warmup + s + 1) * ntr]
            e0.record(stream)
            sv.run(tr, K, dmask, stream=stream.cuda_stream)
            e1.record(stream)
            stream.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
    sieve_pairs_s = ntr * K * K * len(times) / max_over_ranks(sum(times)) * world
    # compulsory HBM bytes of one triple: the prime list read once, the mask written once
    sieve_bytes = 4 * len(primes) + pfb200.mask_bytes(K)
    sieve_gbs = sieve_bytes * ntr * len(times) / max_over_ranks(sum(times)) / 1e9
    # Phase-0 periodic table (primes below 1e4) built on the device, applied per triple
    p0 = pfb200.Phase0(primes[primes < 10000], dev)
    p0_info = p0.info()
    p0_abc = sieve_triples(4096)
    d_p0 = torch.zeros(len(p0_abc) * 313, dtype=torch.int32, device="cuda")
    with torch.cuda.stream(stream):
        p0.apply(p0_abc, d_p0, stream=stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        p0.apply(p0_abc, d_p0, stream=stream.cuda_stream)
        e1.record(stream)
        stream.synchronize()
    phase0 = {"build_s": p0_info["build_seconds"], "masks": p0_info["masks"], "primes": p0_info["primes"],
              "table_gb": p0_info["table_bytes"] / 1e9,
              "apply_triples_per_s": len(p0_abc) / (e0.elapsed_time(e1) / 1e3)}
    p0.close()
    del d_p0
    t = pfb200.GpuTiming()
    dropin_words = pfb200.trial_div_gpu(primes, *abc1, None, t)
    t0 = time.perf_counter()
    for _ in range(3):
        pfb200.trial_div_gpu(primes, *abc1, None, t)
    dropin_s = (time.perf_counter() - t0) / 3
    ref_gpu_sieve = reference_gpu_sieve(primes, abc1, dropin_words) if rank == 0 and not args.no_cpu else None

    # --- Miller-Rabin: resident batch ---------------------------------------
    pairs = uniform_batch_pairs(survivors, seed=replicas.rank_seed(1, rank))  # each rank its own batch
    cands = [pfb200.build_candidate(*abc1, k, j, rev) for (k, j) in pairs for rev in (False, True)]
    sq_per_test = statistics.mean([(N - 1).bit_length() for N in cands])  # bits(d) + 1 check, s = 1
    eng = pfb200.MillerRabin(dev)
    # per-length tuning of the persistent kernel (quantum, steps per launch)
    tune = eng.autotune(14, 15)
    autotune = {"chosen": {str(k): {"quantum": v[0], "chunk": v[1]} for k, v in tune["chosen"].items()},
                "tried": [[r["logl"], r["quantum"], r["chunk"], round(r["squarings_per_s_1"]),
                           round(r["squarings_per_s_2"])] for r in tune["tried"]],
                "columns": "logl, quantum, chunk, squarings/s at 1 and at 2 candidates per SM",
                "fixed": {"lengths": "powers of two 2^8..2^15 (the NTT primes have no factor 3 in p - 1)",
                          "radix": "16 (remainder pass 2, 4 or 8)",
                          "product_form": "one length-L square up to 2^14, cyclic and negacyclic "
                                          "halves at 2^15 (shared-memory capacity)",
                          "candidates_per_cta": "1 (512 threads x 128 registers fill the register file)",
                          "cluster": "1"}}
    batch = pfb200.MRBatch(eng, cands, 2)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    chunk = args.chunk
    tuned_chunk = eng.tuning(14)[1]
    launches_per_step = (chunk + tuned_chunk - 1) // tuned_chunk
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            batch.advance(chunk, stream.cuda_stream)
        stream.synchronize()
        barrier()
        times = []
        done0 = pfb200.batch_steps_done(batch)
        with ClockSampler(dev) as clocks:
            for _ in range(args.steps):
                flush.fill_(1)  # L2 flush between timed steps (outside the events)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                batch.advance(chunk, stream.cuda_stream)
                e1.record(stream)
                stream.synchronize()
                times.append(e0.elapsed_time(e1) / 1e3)
        done1 = pfb200.batch_steps_done(batch)
        barrier()
    t_mr = max_over_ranks(sum(times))
    n = len(cands)
    squarings = done1 - done0  # steps the device executed in the timed launches
    tests_s = squarings / sq_per_test / t_mr * world
    ms_per_step = 1e3 * t_mr / args.steps
    batch.close()

    # plain form: one candidate per call, through the C ABI call a drop-in
    # caller makes (pfb_mr_test on one number: host set-up, upload, the whole
    # test, read-back)
    barrier()
    t0 = time.perf_counter()
    pv, _ = eng.test(cands[:1], 2, residues=True)
    torch.cuda.synchronize()
    plain_s = max_over_ranks(time.perf_counter() - t0)
    plain_tests_s = 1.0 / plain_s

    # uneven batch: 512 candidates of 50 000 - 100 000 digits resident at once,
    # every length advanced by the same persistent launches
    uneven = None
    if not args.no_uneven:
        tup = uneven_tuples(512)
        ucands = [pfb200.build_candidate(*t) for t in tup]
        ub = pfb200.MRBatch(eng, ucands, 2)
        with torch.cuda.stream(stream):
            ub.advance(64, stream.cuda_stream)
            stream.synchronize()
            barrier()
            d0 = pfb200.batch_steps_done(ub)
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ub.advance(256, stream.cuda_stream)
            e1.record(stream)
            stream.synchronize()
            d1 = pfb200.batch_steps_done(ub)
        ub.close()
        t_u = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        mean_bits = statistics.mean(N.bit_length() for N in ucands)
        uneven = {"value": (d1 - d0) / t_u / mean_bits * world, "unit": "tests/s",
                  "candidates": len(ucands), "mean_bits": mean_bits,
                  "digits": [min(t[0] for t in tup), max(t[0] for t in tup)],
                  "squarings_per_s": (d1 - d0) / t_u, "ms_per_step": 1e3 * t_u,
                  "workload": "512 tuples, splitmix64 seed 2: a ~ U[50000,100000], c ~ U[100,1000], "
                              "b ~ U[c+1,a-1], k,j ~ U[1,9999], N or rev(N); 256 squarings each per step"}

    # roofline of the squaring kernel
    peak_lo, peak_hi = pfb200.measure_int32_peak(dev)
    digits = len(str(cands[0]))
    ref_mults = ref_modmuls_per_squaring(digits) * SQ_PER_MODMUL
    achieved = squarings / t_mr * ref_mults  # INT32 multiplies / s (one GPU)
    roofline = {"bound": "int32", "achieved": achieved / 1e12, "peak": peak_lo / 1e12, "unit": "Tmul/s",
                "frac": achieved / peak_lo,
                # DRAM bytes (read + write) of one timed launch of this workload, from one ncu
                # capture of this build (see PERSIST_LAUNCH_DRAM_BYTES); the quantum of that
                # capture and this run's are both reported
                "traffic": PERSIST_LAUNCH_DRAM_BYTES if chunk == 1024 and n == 256 else None,
                "traffic_source": "ncu capture of this build's timed launch (profiles/"
                                  "persist_kernel_uniform_batch_dram.txt), %d-step quanta" % PERSIST_LAUNCH_DRAM_QUANTUM,
                "quantum": eng.tuning(14)[0],
                "peak_source": "measured live: pfb_measure_int32_peak (mul.lo)",
                "mul_hi_peak": peak_hi / 1e12,
                "work": "%d INT32 multiplies per squaring (reference structure at %d digits)" % (ref_mults, digits)}

    # --- serving: continuous batching under Poisson arrivals ---------------
    serving = None
    serve_secs = args.serve_secs if args.serve_secs is not None else (180.0 if world == 1 else 0.0)
    if serve_secs > 0:
        import random
        rng = random.Random(3)
        # requests: N and rev(N) as separate requests, a ~ U[50000, 100000], c ~ U[100, 1000],
        # b ~ U[c+1, a-1] (redrawn while a-b-lk < 2 or b-c <= lj), k, j ~ U[1, 9999]
        def draw():
            return pfb200.build_candidate(*serving_draw(rng))
        props = torch.cuda.get_device_properties(dev)
        # one resident request per SM: a request's squarings then run on an SM
        # of their own (time-to-verdict = its sequential squaring time), and the
        # device's throughput is that of two per SM (the autotuner's columns)
        resident = props.multi_processor_count
        # served capacity on this request mix: a resident batch of `resident`
        # draws, squarings/s over its mean exponent length
        mix = [draw() for _ in range(resident)]
        mb = pfb200.MRBatch(eng, mix, 2)
        with torch.cuda.stream(stream):
            mb.advance(128, stream.cuda_stream)
            stream.synchronize()
            d0 = pfb200.batch_steps_done(mb)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            mb.advance(512, stream.cuda_stream)
            e1.record(stream)
            stream.synchronize()
            d1 = pfb200.batch_steps_done(mb)
        mb.close()
        cap_tests_s = (d1 - d0) / (e0.elapsed_time(e1) / 1e3) / statistics.mean(N.bit_length() for N in mix)
        rate = args.serve_load * cap_tests_s
        srv = pfb200.MRServer(eng, max_resident=resident, hbm_budget_bytes=150 * 10**9, chunk_steps=256)
        t_start = time.perf_counter()
        next_t, tag, lat, done_in_window = 0.0, 0, [], 0
        with ClockSampler(dev) as serve_clocks:
            while time.perf_counter() - t_start < serve_secs:
                now = time.perf_counter() - t_start
                while next_t <= now:
                    srv.submit(draw(), tag)
                    tag += 1
                    next_t += rng.expovariate(rate)
                for r in srv.poll(256, 50):
                    lat.append(r["done_s"] - r["submit_s"])
            done_in_window = len(lat)
            t_drain = time.perf_counter()
            while len(lat) < tag and time.perf_counter() - t_drain < args.serve_drain:
                for r in srv.poll(256, 200):
                    lat.append(r["done_s"] - r["submit_s"])
        drain_s = time.perf_counter() - t_drain
        st = srv.stats()
        srv.close()
        lat.sort()
        pct = (lambda q: lat[min(len(lat) - 1, int(q * len(lat)))] if lat else None)
        serving = {"arrival_seconds": serve_secs, "drain_seconds": drain_s, "arrival_rate_per_s": rate,
                   "submitted": tag, "completed": len(lat), "tests_per_s": done_in_window / serve_secs,
                   "p50_s": pct(0.50), "p99_s": pct(0.99), "max_s": lat[-1] if lat else None,
                   "resident_at_end": st["resident"], "queued_at_end": st["queued"], "launches": st["launches"],
                   "capacity_tests_per_s": cap_tests_s, "max_resident": resident,
                   "hbm_budget_bytes": 150 * 10**9, "clocks": serve_clocks.summary(),
                   "latency_over": "every request submitted in the arrival window (arrival to verdict), "
                                   "after the drain; tests_per_s counts verdicts inside the window",
                   "workload": "Poisson arrivals (seed 3) of N / rev(N), a ~ U[50000,100000], "
                               "k,j ~ U[1,9999], at %.2fx the estimated capacity" % args.serve_load}

    # --- e2e through the C ABI ---------------------------------------------
    e2e = None
    if not args.no_e2e:
        props = torch.cuda.get_device_properties(dev)
        nb = args.e2e_batch or len(cands)
        sub = cands[:nb]
        barrier()
        t0 = time.perf_counter()
        ver, res = eng.test(sub, 2, residues=True)
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t0)
        h2d = sum(2 * ((N.bit_length() + 15) // 16) for N in sub)
        d2h = len(sub) + sum(2 * ((N.bit_length() + 15) // 16) for N in sub)
        e2e = {"value": len(sub) / dt * world, "unit": "tests/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "candidates": len(sub), "seconds": dt,
               "verdicts": {"probable_prime": int(sum(1 for v in ver if v == 1)), "composite":
                            int(sum(1 for v in ver if v == 0))}}
        if args.e2e_breakdown:
            e2e["breakdown"] = e2e_breakdown(pfb200, torch, eng, sub)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC,
        "value": tests_s, "unit": "tests/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "candidates": n, "squarings_per_step": chunk, "squarings_per_test": sq_per_test,
                   "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas"},
        "plain": {"value": plain_tests_s, "unit": "tests/s", "seconds": plain_s,
                  "form": "one candidate per call: pfb_mr_test on one 50 000-digit number from host limbs"},
        "served_over_plain": tests_s / world / plain_tests_s,
        "uneven": uneven,
        "autotune": autotune,
        "phase0": phase0,
        "sieve": {"value": sieve_pairs_s, "unit": "pairs/s", "K": K, "triples_per_step": ntr,
                  "ms_per_triple": 1e3 / (sieve_pairs_s / world / (K * K)),
                  "hbm_compulsory_gbs": sieve_gbs, "hbm_compulsory_bytes_per_triple": sieve_bytes,
                  "dropin_100x100_s": dropin_s, "dropin_timing": {"upload": t.upload, "kernel": t.kernel,
                                                                  "download": t.download},
                  "reference_gpu_100x100": ref_gpu_sieve},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "cpu_baseline_sieve": cpu_sieve,
        "serving": serving,
        "clocks": clocks.summary(),
        "e2e": e2e,
        "gpu_launches": args.steps * launches_per_step,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
