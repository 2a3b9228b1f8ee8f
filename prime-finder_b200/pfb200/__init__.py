"""Python binding of the prime-finder B200 engine (ctypes over the C ABI).

The engine is the shared library ``prime-finder_b200/lib/libpfb200.so``
built from ``prime-finder_b200/csrc`` (sm_100a CUDA + C ABI).  This module
only marshals arguments; every computation runs in the library.  If the
library is missing, the first call into it raises ImportError: there is no
CPU fallback.

Device buffers may be given as integers (raw device pointers) or as any
object with ``data_ptr()`` (e.g. a CUDA ``torch.Tensor``).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence, Tuple

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libpfb200.so")

PFB_OK = 0
PFB_E_CUDA = -1
PFB_E_ARG = -2
PFB_E_NOMEM = -3
PFB_E_CAPACITY = -4
PFB_E_TIMEOUT = -5
PFB_E_STATE = -6

SIEVE_OR = 1
SIEVE_MASK_HOST = 2
SIEVE_MAX_K = 9999


class PfbError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where} failed with code {code}: {last_error()}")


_lib = None


def lib() -> C.CDLL:
    """Load libpfb200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() "
                              "or `make -C prime-finder_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        u32p = C.POINTER(C.c_uint32)
        ll = C.c_longlong
        L.pfb_last_error.restype = C.c_char_p
        L.pfb_sieve_mask_bytes.argtypes = [C.c_int]
        L.pfb_sieve_mask_bytes.restype = C.c_size_t
        L.pfb_sieve_create.argtypes = [C.POINTER(vp), u32p, C.c_uint32, C.c_int]
        L.pfb_sieve_create.restype = C.c_int
        L.pfb_sieve_destroy.argtypes = [vp]
        L.pfb_sieve_destroy.restype = None
        L.pfb_sieve_run.argtypes = [vp, C.POINTER(ll), C.c_int, C.c_int, vp, C.c_uint, vp]
        L.pfb_sieve_run.restype = C.c_int
        L.pfb_sieve_survivors.argtypes = [vp, vp, C.c_int, vp, C.c_uint32, u32p, vp]
        L.pfb_sieve_survivors.restype = C.c_int
        L.trial_div_gpu_grid.argtypes = [u32p, C.c_uint32, C.POINTER(ll), C.c_int, C.c_int,
                                         vp, C.c_uint]
        L.trial_div_gpu_grid.restype = C.c_int
        L.trial_div_gpu.argtypes = [vp, ll, ll, ll, u32p, vp]
        L.trial_div_gpu.restype = C.c_int
        L.cuda_get_device_count.restype = C.c_int
        L.cuda_set_device.argtypes = [C.c_int]
        L.cuda_set_device.restype = C.c_int
        _lib = L
    return _lib


def last_error() -> str:
    if _lib is None:
        return ""
    s = _lib.pfb_last_error()
    return s.decode() if s else ""


def _check(rc: int, where: str) -> None:
    if rc != PFB_OK:
        raise PfbError(rc, where)


def _dptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    return int(x.data_ptr())


def _u32(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _abc_array(abc: Sequence[Tuple[int, int, int]]):
    flat = np.ascontiguousarray(np.asarray(abc, dtype=np.int64).reshape(-1))
    return flat, flat.ctypes.data_as(C.POINTER(C.c_longlong)), len(flat) // 3


# ------------------------------------------------------------------ sieve ---

def mask_bytes(K: int) -> int:
    return int(lib().pfb_sieve_mask_bytes(K))


class PrimeList(C.Structure):
    """prime_list_t (prime_list.h): { uint32_t *primes; uint32_t count; }"""
    _fields_ = [("primes", C.POINTER(C.c_uint32)), ("count", C.c_uint32)]


class GpuTiming(C.Structure):
    """gpu_timing_t (trial_div.h): upload / kernel / download seconds."""
    _fields_ = [("upload", C.c_double), ("kernel", C.c_double), ("download", C.c_double)]


def trial_div_gpu(primes: np.ndarray, a: int, b: int, c: int,
                  sieve_bits: Optional[np.ndarray] = None,
                  timing: Optional[GpuTiming] = None) -> np.ndarray:
    """Drop-in ``trial_div_gpu`` (100 x 100 grid, 313 uint32 words, OR-in)."""
    primes = np.ascontiguousarray(primes, dtype=np.uint32)
    if sieve_bits is None:
        sieve_bits = np.zeros(313, dtype=np.uint32)
    assert sieve_bits.dtype == np.uint32 and sieve_bits.size >= 313
    pl = PrimeList(_u32(primes), len(primes))
    rc = lib().trial_div_gpu(C.addressof(pl), a, b, c, _u32(sieve_bits),
                             C.addressof(timing) if timing is not None else None)
    if rc != 0:
        raise PfbError(rc, "trial_div_gpu")
    return sieve_bits


def trial_div_gpu_grid(primes: np.ndarray, abc, K: int,
                       mask: Optional[np.ndarray] = None, or_in: bool = False) -> np.ndarray:
    """Stateless wide-grid sieve with host buffers; returns the packed masks."""
    primes = np.ascontiguousarray(primes, dtype=np.uint32)
    flat, pabc, n = _abc_array(abc)
    blk = mask_bytes(K)
    if mask is None:
        mask = np.zeros(blk * n, dtype=np.uint8)
    assert mask.nbytes >= blk * n and mask.flags.c_contiguous
    rc = lib().trial_div_gpu_grid(_u32(primes), len(primes), pabc, n, K,
                                  mask.ctypes.data, SIEVE_OR if or_in else 0)
    _check(rc, "trial_div_gpu_grid")
    return mask


class Sieve:
    """A sieve context: the prime list resident in device memory."""

    def __init__(self, primes: np.ndarray, device: int = 0):
        primes = np.ascontiguousarray(primes, dtype=np.uint32)
        h = C.c_void_p()
        _check(lib().pfb_sieve_create(C.byref(h), _u32(primes), len(primes), device),
               "pfb_sieve_create")
        self._h = h
        self.device = device
        self.n_primes = len(primes)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pfb_sieve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, abc, K: int, mask=None, or_in: bool = False, stream: int = 0):
        """Sieve triples into ``mask``: a host ``np.uint8`` array (synchronous) or
        a device buffer (asynchronous on ``stream``).  Returns the mask."""
        flat, pabc, n = _abc_array(abc)
        flags = SIEVE_OR if or_in else 0
        if mask is None or isinstance(mask, np.ndarray):
            if mask is None:
                mask = np.zeros(mask_bytes(K) * n, dtype=np.uint8)
            assert mask.nbytes >= mask_bytes(K) * n
            rc = lib().pfb_sieve_run(self._h, pabc, n, K, mask.ctypes.data,
                                     flags | SIEVE_MASK_HOST, stream or None)
        else:
            rc = lib().pfb_sieve_run(self._h, pabc, n, K, _dptr(mask), flags, stream or None)
        _check(rc, "pfb_sieve_run")
        return mask

    def survivors(self, d_mask, K: int, d_out, cap: int, stream: int = 0) -> int:
        cnt = C.c_uint32(0)
        rc = lib().pfb_sieve_survivors(self._h, _dptr(d_mask), K, _dptr(d_out), cap,
                                       C.byref(cnt), stream or None)
        if rc not in (PFB_OK, PFB_E_CAPACITY):
            _check(rc, "pfb_sieve_survivors")
        return int(cnt.value)


def unpack_mask(mask: np.ndarray, K: int) -> np.ndarray:
    """Packed mask block -> bool array [K, K] (True = eliminated)."""
    bits = np.unpackbits(np.asarray(mask, dtype=np.uint8)[: (K * K + 7) // 8], bitorder="little")
    return bits[: K * K].reshape(K, K).astype(bool)


# ------------------------------------------------------------ Miller-Rabin ---

MR_MAX_BITS = 22 * 16384 - 36


class _Number(C.Structure):
    """pfb_mr_number_t: { const uint16_t *limbs; int n_limbs; }"""
    _fields_ = [("limbs", C.POINTER(C.c_uint16)), ("n_limbs", C.c_int)]


def int_to_limbs16(x: int) -> np.ndarray:
    n = max(1, (x.bit_length() + 15) // 16)
    return np.frombuffer(x.to_bytes(2 * n, "little"), dtype="<u2").copy()


def limbs16_to_int(a: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(a, dtype="<u2").tobytes(), "little")


def _numbers(xs):
    arrs = [x if isinstance(x, np.ndarray) else int_to_limbs16(int(x)) for x in xs]
    arrs = [np.ascontiguousarray(a, dtype=np.uint16) for a in arrs]
    st = (_Number * len(arrs))()
    for i, a in enumerate(arrs):
        st[i].limbs = a.ctypes.data_as(C.POINTER(C.c_uint16))
        st[i].n_limbs = len(a)
    return st, arrs


class TuneRow(C.Structure):
    """pfb_mr_tune_t"""
    _fields_ = [("logl", C.c_int), ("quantum", C.c_int), ("chunk", C.c_int), ("squarings_per_s_1", C.c_double),
                ("squarings_per_s_2", C.c_double)]


def _mr_lib():
    L = lib()
    if not hasattr(L, "_mr_ready"):
        vp = C.c_void_p
        L.pfb_mr_create.argtypes = [C.POINTER(vp), C.c_int]
        L.pfb_mr_create.restype = C.c_int
        L.pfb_mr_destroy.argtypes = [vp]
        L.pfb_mr_destroy.restype = None
        L.pfb_mr_test.argtypes = [vp, C.POINTER(_Number), C.c_int, C.c_uint32,
                                  C.POINTER(C.c_int8), C.POINTER(C.c_uint16), C.c_int]
        L.pfb_mr_test.restype = C.c_int
        L.pfb_mr_powm.argtypes = [vp, C.POINTER(_Number), C.c_int, C.c_uint32,
                                  C.POINTER(_Number), C.POINTER(C.c_uint16), C.c_int]
        L.pfb_mr_powm.restype = C.c_int
        for fn in (L.pfb_mr_lucas, L.pfb_mr_bpsw):
            fn.argtypes = [vp, C.POINTER(_Number), C.c_int, C.POINTER(C.c_int8)]
            fn.restype = C.c_int
        L.pfb_mr_autotune.argtypes = [vp, C.c_int, C.c_int, C.POINTER(TuneRow), C.c_int, C.POINTER(C.c_int)]
        L.pfb_mr_autotune.restype = C.c_int
        L.pfb_mr_get_tuning.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.pfb_mr_get_tuning.restype = C.c_int
        L.pfb_mr_test_cost.argtypes = [C.POINTER(C.c_uint16), C.c_int]
        L.pfb_mr_test_cost.restype = C.c_longlong
        L._mr_ready = True
    return L


class MillerRabin:
    """Batched strong probable-prime tests on one GPU (pfb_mr_* C ABI)."""

    def __init__(self, device: int = 0):
        L = _mr_lib()
        h = C.c_void_p()
        _check(L.pfb_mr_create(C.byref(h), device), "pfb_mr_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _mr_lib().pfb_mr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def test(self, numbers, base: int = 2, residues: bool = True):
        """Returns (verdicts, residues): verdict 1 = probable prime, 0 =
        composite, -1 = invalid input; residue = base^d mod N (N-1 = 2^s d)."""
        st, keep = _numbers(numbers)
        n = len(keep)
        ver = np.zeros(n, dtype=np.int8)
        stride = max(len(a) for a in keep)
        res = np.zeros(n * stride, dtype=np.uint16) if residues else None
        rc = _mr_lib().pfb_mr_test(self._h, st, n, base, ver.ctypes.data_as(C.POINTER(C.c_int8)),
                                   res.ctypes.data_as(C.POINTER(C.c_uint16)) if residues else None,
                                   stride)
        _check(rc, "pfb_mr_test")
        out = None
        if residues:
            out = [limbs16_to_int(res[i * stride:(i + 1) * stride]) for i in range(n)]
        return ver.tolist(), out

    def _verdicts(self, fn, name, numbers):
        st, keep = _numbers(numbers)
        ver = np.zeros(len(keep), dtype=np.int8)
        _check(fn(self._h, st, len(keep), ver.ctypes.data_as(C.POINTER(C.c_int8))), name)
        return ver.tolist()

    def lucas(self, numbers):
        """Strong Lucas test (Selfridge's parameters) per number (pfb_mr_lucas):
        1 strong Lucas probable prime, 0 composite, -1 invalid."""
        return self._verdicts(_mr_lib().pfb_mr_lucas, "pfb_mr_lucas", numbers)

    def bpsw(self, numbers):
        """Baillie-PSW per number (pfb_mr_bpsw): 1 probable prime, 0 composite,
        -1 too long."""
        return self._verdicts(_mr_lib().pfb_mr_bpsw, "pfb_mr_bpsw", numbers)

    def autotune(self, logl_lo: int = 14, logl_hi: int = 15):
        """Tune (quantum, chunk) of the persistent kernel per transform length
        (pfb_mr_autotune).  Returns {"tried": [...], "chosen": {logl: (q, c)}}."""
        L = _mr_lib()
        rows = (TuneRow * 64)()
        n = C.c_int(0)
        _check(L.pfb_mr_autotune(self._h, logl_lo, logl_hi, rows, 64, C.byref(n)), "pfb_mr_autotune")
        tried = [{"logl": r.logl, "quantum": r.quantum, "chunk": r.chunk,
                  "squarings_per_s_1": r.squarings_per_s_1, "squarings_per_s_2": r.squarings_per_s_2}
                 for r in rows[:n.value]]
        return {"tried": tried, "chosen": {lg: self.tuning(lg) for lg in range(logl_lo, logl_hi + 1)}}

    def tuning(self, logl: int):
        q, c = C.c_int(0), C.c_int(0)
        _check(_mr_lib().pfb_mr_get_tuning(self._h, logl, C.byref(q), C.byref(c)), "pfb_mr_get_tuning")
        return q.value, c.value

    def powm(self, numbers, exps, base: int = 2):
        st, keep = _numbers(numbers)
        se, keep_e = _numbers(exps)
        n = len(keep)
        stride = max(len(a) for a in keep)
        res = np.zeros(n * stride, dtype=np.uint16)
        rc = _mr_lib().pfb_mr_powm(self._h, st, n, base, se,
                                   res.ctypes.data_as(C.POINTER(C.c_uint16)), stride)
        _check(rc, "pfb_mr_powm")
        return [limbs16_to_int(res[i * stride:(i + 1) * stride]) for i in range(n)]


def _batch_lib():
    L = _mr_lib()
    if not hasattr(L, "_batch_ready"):
        vp = C.c_void_p
        L.pfb_mr_batch_create.argtypes = [vp, C.POINTER(_Number), C.c_int, C.c_uint32, C.POINTER(vp)]
        L.pfb_mr_batch_create.restype = C.c_int
        L.pfb_mr_batch_advance.argtypes = [vp, C.c_int, vp]
        L.pfb_mr_batch_advance.restype = C.c_int
        L.pfb_mr_batch_pending.argtypes = [vp, C.POINTER(C.c_int)]
        L.pfb_mr_batch_pending.restype = C.c_int
        L.pfb_mr_batch_steps_left.argtypes = [vp]
        L.pfb_mr_batch_steps_left.restype = C.c_longlong
        L.pfb_mr_batch_results.argtypes = [vp, C.POINTER(C.c_int8), C.POINTER(C.c_uint16), C.c_int]
        L.pfb_mr_batch_results.restype = C.c_int
        L.pfb_mr_batch_destroy.argtypes = [vp]
        L.pfb_mr_batch_destroy.restype = None
        L.pfb_measure_int32_peak.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.pfb_measure_int32_peak.restype = C.c_int
        L._batch_ready = True
    return L


class MRBatch:
    """Candidates resident on the GPU, advanced step by step (pfb_mr_batch_*)."""

    def __init__(self, engine: "MillerRabin", numbers, base: int = 2):
        L = _batch_lib()
        st, self._keep = _numbers(numbers)
        h = C.c_void_p()
        _check(L.pfb_mr_batch_create(engine._h, st, len(self._keep), base, C.byref(h)),
               "pfb_mr_batch_create")
        self._h = h
        self.n = len(self._keep)

    def advance(self, steps: int, stream: int = 0) -> None:
        _check(_batch_lib().pfb_mr_batch_advance(self._h, steps, stream or None), "pfb_mr_batch_advance")

    def steps_left(self) -> int:
        return int(_batch_lib().pfb_mr_batch_steps_left(self._h))

    def pending(self) -> int:
        c = C.c_int(0)
        _check(_batch_lib().pfb_mr_batch_pending(self._h, C.byref(c)), "pfb_mr_batch_pending")
        return int(c.value)

    def results(self, residues: bool = False):
        ver = np.zeros(self.n, dtype=np.int8)
        stride = max(len(a) for a in self._keep)
        res = np.zeros(self.n * stride, dtype=np.uint16) if residues else None
        rc = _batch_lib().pfb_mr_batch_results(
            self._h, ver.ctypes.data_as(C.POINTER(C.c_int8)),
            res.ctypes.data_as(C.POINTER(C.c_uint16)) if residues else None, stride)
        if rc not in (PFB_OK, PFB_E_STATE):
            _check(rc, "pfb_mr_batch_results")
        out = None
        if residues:
            out = [limbs16_to_int(res[i * stride:(i + 1) * stride]) for i in range(self.n)]
        return ver.tolist(), out

    def close(self):
        if getattr(self, "_h", None):
            _batch_lib().pfb_mr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def radix16_forms(engine: "MillerRabin", ctas: int = 592, reps: int = 20) -> dict:
    """One radix-16 transform pass in its butterfly form and as a tensor-core
    byte-plane product (pfb_mr_radix16_forms): per-launch times, output
    mismatches between the two forms, the tensor form's timeout flag."""
    L = _mr_lib()
    f = L.pfb_mr_radix16_forms
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                  C.POINTER(C.c_longlong), C.POINTER(C.c_int)]
    f.restype = C.c_int
    tb, tt, bad, err = C.c_double(), C.c_double(), C.c_longlong(), C.c_int()
    _check(f(engine._h, ctas, reps, C.byref(tb), C.byref(tt), C.byref(bad), C.byref(err)), "pfb_mr_radix16_forms")
    return {"ms_butterfly": tb.value, "ms_tensor": tt.value, "mismatches": bad.value, "tensor_timeout": err.value}


def measure_int32_peak(device: int = 0):
    """(mul.lo ops/s, mul.hi ops/s) sustained on `device`."""
    lo, hi = C.c_double(0), C.c_double(0)
    _check(_batch_lib().pfb_measure_int32_peak(device, C.byref(lo), C.byref(hi)), "pfb_measure_int32_peak")
    return lo.value, hi.value


# ----------------------------------------------------------- candidates ---

def ndigits(x: int) -> int:
    """Decimal digits of a small non-negative integer (k or j)."""
    return len(str(x))


def rev_digits(x: int, lx: int) -> int:
    return int(str(x).zfill(lx)[::-1])


def build_candidate(a: int, b: int, c: int, k: int, j: int, rev: bool = False) -> int:
    """N = 10^a - k 10^b - j 10^c - 1, or rev(N) = 10^a - rev(k) 10^(a-b-lk)
    - rev(j) 10^(a-c-lj) - 1 (miller_rabin.c:56-99)."""
    if rev:
        lk, lj = ndigits(k), ndigits(j)
        return 10 ** a - rev_digits(k, lk) * 10 ** (a - b - lk) - rev_digits(j, lj) * 10 ** (a - c - lj) - 1
    return 10 ** a - k * 10 ** b - j * 10 ** c - 1


# ----------------------------------------------------------------- serving ---

class ServerConfig(C.Structure):
    """pfb_mr_server_config_t"""
    _fields_ = [("max_resident", C.c_int), ("hbm_budget_bytes", C.c_size_t), ("chunk_steps", C.c_int),
                ("base", C.c_uint32), ("prep_threads", C.c_int)]


class ServerResult(C.Structure):
    """pfb_mr_result_t"""
    _fields_ = [("tag", C.c_uint64), ("verdict", C.c_int8), ("submit_s", C.c_double),
                ("admit_s", C.c_double), ("done_s", C.c_double)]


class ServerStats(C.Structure):
    """pfb_mr_server_stats_t"""
    _fields_ = [("submitted", C.c_longlong), ("admitted", C.c_longlong), ("completed", C.c_longlong),
                ("launches", C.c_longlong), ("steps_retired", C.c_longlong), ("resident", C.c_int),
                ("queued", C.c_int), ("error", C.c_int), ("bytes_in_use", C.c_size_t),
                ("bytes_owned", C.c_size_t)]


def _server_lib():
    L = _batch_lib()
    if not hasattr(L, "_server_ready"):
        vp = C.c_void_p
        L.pfb_mr_server_create.argtypes = [vp, C.POINTER(ServerConfig), C.POINTER(vp)]
        L.pfb_mr_server_create.restype = C.c_int
        L.pfb_mr_server_submit.argtypes = [vp, C.POINTER(C.c_uint16), C.c_int, C.c_uint64,
                                           C.POINTER(C.c_uint16), C.c_int]
        L.pfb_mr_server_submit.restype = C.c_int
        L.pfb_mr_server_poll.argtypes = [vp, C.POINTER(ServerResult), C.c_int, C.c_int]
        L.pfb_mr_server_poll.restype = C.c_int
        L.pfb_mr_server_stats.argtypes = [vp, C.POINTER(ServerStats)]
        L.pfb_mr_server_stats.restype = C.c_int
        L.pfb_mr_server_destroy.argtypes = [vp]
        L.pfb_mr_server_destroy.restype = None
        L.pfb_mr_server_inject_alloc_failures.argtypes = [vp, C.c_int]
        L.pfb_mr_server_inject_alloc_failures.restype = C.c_int
        L.pfb_mr_batch_steps_done.argtypes = [vp]
        L.pfb_mr_batch_steps_done.restype = C.c_longlong
        L._server_ready = True
    return L


class MRServer:
    """Continuous-batching strong-test server (pfb_mr_server_* C ABI)."""

    def __init__(self, engine: "MillerRabin", max_resident: int = 0, hbm_budget_bytes: int = 0,
                 chunk_steps: int = 0, base: int = 2, prep_threads: int = 0):
        L = _server_lib()
        self._cfg = ServerConfig(max_resident, hbm_budget_bytes, chunk_steps, base, prep_threads)
        h = C.c_void_p()
        _check(L.pfb_mr_server_create(engine._h, C.byref(self._cfg), C.byref(h)), "pfb_mr_server_create")
        self._h = h
        self._bufs = {}   # tag -> (limbs, residue buffer) kept alive until the result is read

    def submit(self, number, tag: int, residue: bool = False) -> None:
        limbs = number if isinstance(number, np.ndarray) else int_to_limbs16(int(number))
        limbs = np.ascontiguousarray(limbs, dtype=np.uint16)
        res = np.zeros(len(limbs), dtype=np.uint16) if residue else None
        self._bufs[tag] = (limbs, res)
        rc = _server_lib().pfb_mr_server_submit(
            self._h, limbs.ctypes.data_as(C.POINTER(C.c_uint16)), len(limbs), tag,
            res.ctypes.data_as(C.POINTER(C.c_uint16)) if residue else None, len(limbs) if residue else 0)
        _check(rc, "pfb_mr_server_submit")

    def poll(self, cap: int = 64, timeout_ms: int = 100):
        """List of dicts {tag, verdict, submit_s, admit_s, done_s[, residue]}."""
        out = (ServerResult * cap)()
        n = _server_lib().pfb_mr_server_poll(self._h, out, cap, timeout_ms)
        if n < 0:
            raise PfbError(n, "pfb_mr_server_poll")
        res = []
        for i in range(n):
            r = out[i]
            d = {"tag": int(r.tag), "verdict": int(r.verdict), "submit_s": r.submit_s,
                 "admit_s": r.admit_s, "done_s": r.done_s}
            limbs, rb = self._bufs.pop(int(r.tag), (None, None))
            if rb is not None:
                d["residue"] = limbs16_to_int(rb)
            res.append(d)
        return res

    def inject_alloc_failures(self, n: int) -> int:
        """Test hook: the next n slot allocations fail on the host as if the
        device were out of memory; returns the injected failures consumed."""
        rc = _server_lib().pfb_mr_server_inject_alloc_failures(self._h, n)
        if rc < 0:
            raise PfbError(rc, "pfb_mr_server_inject_alloc_failures")
        return rc

    def stats(self) -> dict:
        st = ServerStats()
        _check(_server_lib().pfb_mr_server_stats(self._h, C.byref(st)), "pfb_mr_server_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _server_lib().pfb_mr_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_steps_done(batch: "MRBatch") -> int:
    return int(_server_lib().pfb_mr_batch_steps_done(batch._h))


# ---------------------------------------------------------------- pipeline ---

class Phase2Record(C.Structure):
    """pfb_phase2_record_t"""
    _fields_ = [("a", C.c_longlong), ("b", C.c_longlong), ("c", C.c_longlong), ("k", C.c_int),
                ("j", C.c_int), ("result", C.c_int)]


class PipelineConfig(C.Structure):
    """pfb_pipeline_config_t"""
    _fields_ = [("K", C.c_int), ("triples_per_sieve", C.c_int), ("max_resident", C.c_int),
                ("hbm_budget_bytes", C.c_size_t), ("prep_threads", C.c_int), ("window", C.c_int)]


class PipelineStats(C.Structure):
    """pfb_pipeline_stats_t"""
    _fields_ = [("triples", C.c_longlong), ("survivors", C.c_longlong), ("n_prp", C.c_longlong),
                ("rev_tested", C.c_longlong), ("both_prp", C.c_longlong), ("invalid", C.c_longlong),
                ("sieve_s", C.c_double), ("phase2_s", C.c_double), ("total_s", C.c_double)]


def _pipeline_lib():
    L = _mr_lib()
    if not hasattr(L, "_pipeline_ready"):
        L.pfb_pipeline_run.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong), C.c_int,
                                       C.POINTER(PipelineConfig), C.POINTER(C.c_uint8),
                                       C.POINTER(Phase2Record), C.c_longlong, C.POINTER(C.c_longlong),
                                       C.POINTER(PipelineStats)]
        L.pfb_pipeline_run.restype = C.c_int
        L.pfb_mr_device.argtypes = [C.c_void_p]
        L.pfb_mr_device.restype = C.c_int
        L._pipeline_ready = True
    return L


def pipeline_run(sieve: "Sieve", engine: "MillerRabin", abc, K: int, pre_mask: Optional[np.ndarray] = None,
                 cap: Optional[int] = None, triples_per_sieve: int = 0, max_resident: int = 0,
                 hbm_budget_bytes: int = 0, prep_threads: int = 0, window: int = 0):
    """Sieve the triples on the K x K grid and decide every survivor
    (pfb_pipeline_run).  Returns ([(a, b, c, k, j, result), ...], stats)
    with miller_rabin_test result codes, triple order, k-major."""
    L = _pipeline_lib()
    flat, pabc, n = _abc_array(abc)
    cfg = PipelineConfig(K, triples_per_sieve, max_resident, hbm_budget_bytes, prep_threads, window)
    pm = None
    if pre_mask is not None:
        pre_mask = np.ascontiguousarray(pre_mask, dtype=np.uint8)
        if pre_mask.size < mask_bytes(K) * n:
            raise ValueError("pre_mask holds fewer than n_abc mask blocks")
        pm = pre_mask.ctypes.data_as(C.POINTER(C.c_uint8))
    st = PipelineStats()
    n_out = C.c_longlong(0)
    if cap is None:
        # count first: a zero-capacity call sieves and reports the survivors
        rc = L.pfb_pipeline_run(sieve._h, engine._h, pabc, n, C.byref(cfg), pm, None, 0, C.byref(n_out),
                                C.byref(st))
        if rc not in (PFB_OK, -4):
            raise PfbError(rc, "pfb_pipeline_run")
        cap = n_out.value
    out = (Phase2Record * max(1, cap))()
    _check(L.pfb_pipeline_run(sieve._h, engine._h, pabc, n, C.byref(cfg), pm, out, cap, C.byref(n_out),
                              C.byref(st)), "pfb_pipeline_run")
    recs = [(r.a, r.b, r.c, r.k, r.j, r.result) for r in out[:n_out.value]]
    return recs, {f: getattr(st, f) for f, _ in PipelineStats._fields_}


# ------------------------------------------------------------------ phase 0 ---

def _phase0_lib():
    L = lib()
    if not hasattr(L, "_phase0_ready"):
        vp = C.c_void_p
        L.pfb_phase0_create.argtypes = [C.POINTER(vp), C.POINTER(C.c_uint32), C.c_uint32, C.c_int]
        L.pfb_phase0_create.restype = C.c_int
        L.pfb_phase0_apply.argtypes = [vp, C.POINTER(C.c_longlong), C.c_int, vp, C.c_uint, vp]
        L.pfb_phase0_apply.restype = C.c_int
        L.pfb_phase0_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_size_t),
                                      C.POINTER(C.c_double)]
        L.pfb_phase0_info.restype = C.c_int
        L.pfb_phase0_destroy.argtypes = [vp]
        L.pfb_phase0_destroy.restype = None
        L._phase0_ready = True
    return L


class Phase0:
    """The Phase-0 periodic table in device memory (pfb_phase0_* C ABI)."""

    def __init__(self, small_primes: np.ndarray, device: int = 0):
        small_primes = np.ascontiguousarray(small_primes, dtype=np.uint32)
        h = C.c_void_p()
        _check(_phase0_lib().pfb_phase0_create(C.byref(h), _u32(small_primes), len(small_primes), device),
               "pfb_phase0_create")
        self._h = h

    def info(self) -> dict:
        n, m, b, s = C.c_int(0), C.c_longlong(0), C.c_size_t(0), C.c_double(0)
        _check(_phase0_lib().pfb_phase0_info(self._h, C.byref(n), C.byref(m), C.byref(b), C.byref(s)),
               "pfb_phase0_info")
        return {"primes": n.value, "masks": m.value, "table_bytes": b.value, "build_seconds": s.value}

    def apply(self, abc, masks=None, or_in: bool = False, stream: int = 0):
        """313-word masks of the triples: into a host array (returned) or a
        device buffer (asynchronous on stream)."""
        flat, pabc, n = _abc_array(abc)
        flags = SIEVE_OR if or_in else 0
        if masks is None or isinstance(masks, np.ndarray):
            if masks is None:
                masks = np.zeros((n, 313), dtype=np.uint32)
            masks = np.ascontiguousarray(masks, dtype=np.uint32)
            _check(_phase0_lib().pfb_phase0_apply(self._h, pabc, n, masks.ctypes.data, flags | SIEVE_MASK_HOST,
                                                  None), "pfb_phase0_apply")
            return masks
        _check(_phase0_lib().pfb_phase0_apply(self._h, pabc, n, _dptr(masks), flags, stream or None),
               "pfb_phase0_apply")
        return masks

    def close(self):
        if getattr(self, "_h", None):
            _phase0_lib().pfb_phase0_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ formats ---

class Candidate(C.Structure):
    """pfb_candidate_t"""
    _fields_ = [("a", C.c_longlong), ("b", C.c_longlong), ("c", C.c_longlong), ("k", C.c_int), ("j", C.c_int)]


def _formats_lib():
    L = lib()
    if not hasattr(L, "_formats_ready"):
        L.pfb_read_candidates.argtypes = [C.c_char_p, C.POINTER(Candidate), C.c_longlong]
        L.pfb_read_candidates.restype = C.c_longlong
        for fn in (L.pfb_write_phase1, L.pfb_write_phase2):
            fn.argtypes = [C.c_char_p, C.POINTER(Phase2Record), C.c_longlong, C.c_int]
            fn.restype = C.c_longlong
        L._formats_ready = True
    return L


def read_candidates(path: str):
    """[(a, b, c, k, j), ...] of a candidate file (pfb_read_candidates)."""
    L = _formats_lib()
    n = L.pfb_read_candidates(path.encode(), None, 0)
    if n < 0:
        raise PfbError(int(n), "pfb_read_candidates")
    out = (Candidate * max(1, n))()
    L.pfb_read_candidates(path.encode(), out, n)
    return [(r.a, r.b, r.c, r.k, r.j) for r in out[:n]]


def _records(recs):
    arr = (Phase2Record * max(1, len(recs)))()
    for i, r in enumerate(recs):
        arr[i] = Phase2Record(*(list(r[:5]) + [r[5] if len(r) > 5 else 0]))
    return arr


def write_phase1(path: str, recs, append: bool = False) -> int:
    """Survivor lines "a=.. b=.. c=.. k=.. j=.." (pfb_write_phase1)."""
    n = _formats_lib().pfb_write_phase1(path.encode(), _records(recs), len(recs), int(append))
    if n < 0:
        raise PfbError(int(n), "pfb_write_phase1")
    return int(n)


def write_phase2(path: str, recs, append: bool = False) -> int:
    """Hit lines for result 2 / 3 records (pfb_write_phase2)."""
    n = _formats_lib().pfb_write_phase2(path.encode(), _records(recs), len(recs), int(append))
    if n < 0:
        raise PfbError(int(n), "pfb_write_phase2")
    return int(n)
