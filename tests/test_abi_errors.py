"""Every C-ABI entry point rejects invalid arguments with its documented code
and a one-line message, before any CUDA call (so this runs without a GPU).

The reference's entry points return 0 / -1 with a line on stderr
(trial_div.cu:222, miller_rabin.c:76-118); the drop-ins keep that, and the
pfb_* extensions return a negative PFB_E_* code with pfb_last_error() set.
"""
import ctypes as C

import pfb200

E_ARG, E_CAPACITY = pfb200.PFB_E_ARG, pfb200.PFB_E_CAPACITY
NULL = None
FAKE = C.c_void_p(0x1000)  # never dereferenced: every call below fails its checks first


def _lib():
    L = pfb200.lib()
    vp, i, u, ll = C.c_void_p, C.c_int, C.c_uint32, C.c_longlong
    sigs = {
        "pfb_sieve_create": [vp, vp, u, i],
        "pfb_sieve_run": [vp, vp, i, i, vp, C.c_uint, vp],
        "pfb_sieve_survivors": [vp, vp, i, vp, u, vp, vp],
        "pfb_sieve_run_noalloc": [vp, u, ll, ll, ll, i, vp, C.c_uint, vp],
        "trial_div_gpu_grid": [vp, u, vp, i, i, vp, C.c_uint],
        "trial_div_gpu": [vp, ll, ll, ll, vp, vp],
        "miller_rabin_test": [ll, ll, ll, i, i, vp],
        "pfb_mr_create": [vp, i],
        "pfb_mr_test": [vp, vp, i, u, vp, vp, i],
        "pfb_mr_lucas": [vp, vp, i, vp],
        "pfb_mr_bpsw": [vp, vp, i, vp],
        "pfb_mr_powm": [vp, vp, i, u, vp, vp, i],
        "pfb_mr_batch_create": [vp, vp, i, u, vp],
        "pfb_mr_batch_advance": [vp, i, vp],
        "pfb_mr_autotune": [vp, i, i, vp, i, vp],
        "pfb_mr_get_tuning": [vp, i, vp, vp],
        "pfb_mr_server_create": [vp, vp, vp],
        "pfb_mr_server_submit": [vp, vp, i, C.c_uint64, vp, i],
        "pfb_mr_server_poll": [vp, vp, i, i],
        "pfb_pipeline_run": [vp, vp, vp, i, vp, vp, vp, ll, vp, vp],
        "pfb_phase0_create": [vp, vp, u, i],
        "pfb_phase0_apply": [vp, vp, i, vp, C.c_uint, vp],
    }
    for name, args in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    return L


def _err(code, where):
    assert code == E_ARG or code == E_CAPACITY, (where, code)
    msg = pfb200.last_error()
    assert msg, where


def test_sieve_entry_points_reject_bad_arguments():
    L = _lib()
    _err(L.pfb_sieve_create(NULL, NULL, 0, 0), "create: null out")
    _err(L.pfb_sieve_create(FAKE, NULL, 5, 0), "create: primes missing")
    _err(L.pfb_sieve_run(NULL, FAKE, 1, 100, FAKE, 0, NULL), "run: null context")
    _err(L.pfb_sieve_survivors(NULL, FAKE, 100, FAKE, 1, FAKE, NULL), "survivors: null context")
    _err(L.trial_div_gpu_grid(NULL, 5, FAKE, 1, 100, FAKE, 0), "grid: primes missing")
    assert pfb200.mask_bytes(0) == 0 and pfb200.mask_bytes(1) == 4


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch():
    L = _lib()
    assert L.pfb_sieve_run_noalloc(FAKE, 10, 60, 40, 20, 10000, FAKE, 0, NULL) == E_CAPACITY
    assert "9999" in pfb200.last_error()
    assert L.pfb_sieve_run_noalloc(FAKE, 10, 60, 40, 20, 0, FAKE, 0, NULL) == E_CAPACITY
    _err(L.pfb_sieve_run_noalloc(FAKE, 10, -1, 40, 20, 100, FAKE, 0, NULL), "noalloc: negative exponent")
    _err(L.pfb_sieve_run_noalloc(NULL, 10, 60, 40, 20, 100, FAKE, 0, NULL), "noalloc: primes missing")


def test_reference_drop_ins_return_minus_one():
    L = _lib()
    assert L.trial_div_gpu(NULL, 50000, 30000, 100, FAKE, NULL) == -1
    t = (C.c_double * 4)(7, 7, 7, 7)
    assert L.miller_rabin_test(50000, 30000, 100, 0, 5, C.cast(t, C.c_void_p)) == -1
    assert list(t) == [0.0, 0.0, 0.0, 0.0]  # timing cleared, as the reference does
    assert L.miller_rabin_test(50000, 30000, 100, 5, 10000, NULL) == -1


def test_engine_entry_points_reject_bad_arguments():
    L = _lib()
    _err(L.pfb_mr_create(NULL, 0), "mr_create: null out")
    _err(L.pfb_mr_test(NULL, FAKE, 1, 2, FAKE, NULL, 0), "test: null engine")
    _err(L.pfb_mr_test(FAKE, FAKE, 1, 2, FAKE, FAKE, 0), "test: residue stride 0")
    _err(L.pfb_mr_lucas(FAKE, FAKE, 1, NULL), "lucas: no verdict buffer")
    _err(L.pfb_mr_bpsw(NULL, FAKE, 1, FAKE), "bpsw: null engine")
    _err(L.pfb_mr_powm(FAKE, FAKE, 1, 2, NULL, FAKE, 4), "powm: no exponents")
    _err(L.pfb_mr_batch_create(FAKE, FAKE, 1, 2, NULL), "batch_create: null out")
    _err(L.pfb_mr_batch_advance(NULL, 10, NULL), "batch_advance: null batch")
    _err(L.pfb_mr_autotune(FAKE, 7, 15, NULL, 0, NULL), "autotune: length below 2^8")
    _err(L.pfb_mr_autotune(FAKE, 14, 16, NULL, 0, NULL), "autotune: length above 2^15")
    _err(L.pfb_mr_get_tuning(NULL, 14, NULL, NULL), "get_tuning: null engine")
    _err(L.pfb_mr_server_create(NULL, NULL, FAKE), "server_create: null engine")
    _err(L.pfb_mr_server_submit(NULL, FAKE, 1, 0, NULL, 0), "submit: null server")
    _err(L.pfb_mr_server_poll(NULL, FAKE, 1, 0), "poll: null server")


def test_pipeline_and_phase0_reject_bad_arguments():
    L = _lib()
    _err(L.pfb_pipeline_run(NULL, FAKE, FAKE, 1, FAKE, NULL, NULL, 0, FAKE, NULL), "pipeline: null sieve")
    _err(L.pfb_phase0_create(NULL, NULL, 0, 0), "phase0_create: null out")
    _err(L.pfb_phase0_apply(NULL, FAKE, 1, FAKE, 0, NULL), "phase0_apply: null table")
