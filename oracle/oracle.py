"""ctypes front-end to the CPU oracles (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker / the timed CPU
baseline.  The product (``prime-finder_b200``) never imports it.

Two families of libraries are loaded:

* ``liboracle.so`` - our C restatements (``sieve_oracle.c``, ``mr_oracle.c``).
* ``_ref/libref_sieve.so`` / ``_ref/libref_mr.so`` / ``_ref/libref_phase0.so``
  - the reference's own ``trial_div_cpu.c``, ``prime_list.c``,
  ``miller_rabin.c``, ``sieve_table.c`` and ``sieve.c``, compiled unmodified
  by ``oracle/Makefile``.
* ``_ref/libref_trial_div_gpu.so`` - the reference's own GPU sieve
  (``trial_div.cu``), compiled unmodified for sm_100a: the baseline kernel the
  drop-in ``trial_div_gpu`` is timed against.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_lib = None
_ref_sieve = None
_ref_mr = None


def _build_if_missing() -> None:
    if not os.path.exists(os.path.join(HERE, "liboracle.so")):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        _build_if_missing()
        L = C.CDLL(os.path.join(HERE, "liboracle.so"))
        u32p = C.POINTER(C.c_uint32)
        u8p = C.POINTER(C.c_uint8)
        u16p = C.POINTER(C.c_uint16)
        ll = C.c_longlong
        L.oracle_sieve_grid.argtypes = [u32p, C.c_uint32, ll, ll, ll, C.c_int, u8p, C.c_int]
        L.oracle_sieve_grid.restype = None
        L.oracle_sieve_brute.argtypes = [u32p, C.c_uint32, ll, ll, ll, C.c_int, u8p]
        L.oracle_sieve_brute.restype = None
        L.oracle_primes_below.argtypes = [C.c_uint32, u32p, C.c_uint32]
        L.oracle_primes_below.restype = C.c_uint32
        L.oracle_build_candidate.argtypes = [ll, ll, ll, C.c_int, C.c_int, C.c_int, u16p, C.c_int]
        L.oracle_build_candidate.restype = C.c_int
        L.oracle_strong_residue.argtypes = [u16p, C.c_int, C.c_ulong, u16p, C.c_int]
        L.oracle_strong_residue.restype = C.c_int
        L.oracle_strong_test.argtypes = [u16p, C.c_int, C.c_ulong]
        L.oracle_strong_test.restype = C.c_int
        L.oracle_probab_prime.argtypes = [u16p, C.c_int, C.c_int]
        L.oracle_probab_prime.restype = C.c_int
        L.oracle_mulmod.argtypes = [u16p, u16p, u16p, C.c_int, u16p]
        L.oracle_mulmod.restype = C.c_int
        L.oracle_powm.argtypes = [u16p, C.c_int, u16p, C.c_int, u16p, C.c_int, u16p]
        L.oracle_powm.restype = C.c_int
        L.oracle_nextprime.argtypes = [u16p, C.c_int, u16p, C.c_int]
        L.oracle_nextprime.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


# ----------------------------------------------------------------- sieve ----

def mask_bytes(K: int) -> int:
    return (K * K + 7) // 8


def primes_below(limit: int) -> np.ndarray:
    """Odd primes <= limit (2 excluded, as gen_primes.c:119-122 does)."""
    L = lib()
    n = L.oracle_primes_below(limit, None, 0)
    out = np.zeros(max(n, 1), dtype=np.uint32)
    L.oracle_primes_below(limit, _ptr(out, C.c_uint32), n)
    return out[:n]


def sieve_grid(primes: np.ndarray, a: int, b: int, c: int, K: int,
               mask: Optional[np.ndarray] = None, threads: int = 0) -> np.ndarray:
    """Restated trial_div_cpu over a K x K grid; returns the packed mask."""
    primes = np.ascontiguousarray(primes, dtype=np.uint32)
    if mask is None:
        mask = np.zeros(mask_bytes(K), dtype=np.uint8)
    if threads <= 0:
        threads = os.cpu_count() or 1
    lib().oracle_sieve_grid(_ptr(primes, C.c_uint32), len(primes), a, b, c, K,
                            _ptr(mask, C.c_uint8), threads)
    return mask


def sieve_brute(primes: np.ndarray, a: int, b: int, c: int, K: int) -> np.ndarray:
    primes = np.ascontiguousarray(primes, dtype=np.uint32)
    mask = np.zeros(mask_bytes(K), dtype=np.uint8)
    lib().oracle_sieve_brute(_ptr(primes, C.c_uint32), len(primes), a, b, c, K,
                             _ptr(mask, C.c_uint8))
    return mask


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_sieve.so"))


class _PrimeList(C.Structure):
    # prime_list.h: { uint32_t *primes; uint32_t count; }
    _fields_ = [("primes", C.POINTER(C.c_uint32)), ("count", C.c_uint32)]


def ref_trial_div_cpu(primes: np.ndarray, a: int, b: int, c: int,
                      bits: Optional[np.ndarray] = None) -> np.ndarray:
    """The reference's own trial_div_cpu (100 x 100 grid, 313 u32 words)."""
    global _ref_sieve
    if _ref_sieve is None:
        _ref_sieve = C.CDLL(os.path.join(REF_DIR, "libref_sieve.so"))
        _ref_sieve.trial_div_cpu.argtypes = [C.POINTER(_PrimeList), C.c_longlong,
                                             C.c_longlong, C.c_longlong,
                                             C.POINTER(C.c_uint32)]
        _ref_sieve.trial_div_cpu.restype = None
    primes = np.ascontiguousarray(primes, dtype=np.uint32)
    if bits is None:
        bits = np.zeros(313, dtype=np.uint32)
    pl = _PrimeList(_ptr(primes, C.c_uint32), len(primes))
    _ref_sieve.trial_div_cpu(C.byref(pl), a, b, c, _ptr(bits, C.c_uint32))
    return bits


class _GpuTiming(C.Structure):
    # trial_div.h: { double upload, kernel, download; }
    _fields_ = [("upload", C.c_double), ("kernel", C.c_double), ("download", C.c_double)]


_ref_gpu = None


def ref_gpu_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_trial_div_gpu.so"))


def ref_trial_div_gpu(primes: np.ndarray, a: int, b: int, c: int,
                      bits: Optional[np.ndarray] = None):
    """The reference's own trial_div_gpu (trial_div.cu:155-224) on the current
    CUDA device: returns (313 u32 words, rc, {upload, kernel, download} s)."""
    global _ref_gpu
    if _ref_gpu is None:
        _ref_gpu = C.CDLL(os.path.join(REF_DIR, "libref_trial_div_gpu.so"))
        _ref_gpu.trial_div_gpu.argtypes = [C.POINTER(_PrimeList), C.c_longlong, C.c_longlong,
                                           C.c_longlong, C.POINTER(C.c_uint32), C.POINTER(_GpuTiming)]
        _ref_gpu.trial_div_gpu.restype = C.c_int
    primes = np.ascontiguousarray(primes, dtype=np.uint32)
    if bits is None:
        bits = np.zeros(313, dtype=np.uint32)
    pl = _PrimeList(_ptr(primes, C.c_uint32), len(primes))
    t = _GpuTiming()
    rc = _ref_gpu.trial_div_gpu(C.byref(pl), a, b, c, _ptr(bits, C.c_uint32), C.byref(t))
    return bits, rc, {"upload": t.upload, "kernel": t.kernel, "download": t.download}


class _SieveTable(C.Structure):
    # sieve_table.h: { sieve_entry_t *entries; int n; uint32_t *flat_data; size_t flat_size; int shared; }
    _fields_ = [("entries", C.c_void_p), ("n", C.c_int), ("flat_data", C.c_void_p),
                ("flat_size", C.c_size_t), ("shared", C.c_int)]


def ref_phase0_masks(small_primes: np.ndarray, abc) -> np.ndarray:
    """The reference's own Phase 0: sieve_table_build over small_primes, then
    sieve_apply per triple; returns [len(abc), 313] u32 masks.  Builds the
    whole table (4 GB for the primes below 1e4)."""
    L = C.CDLL(os.path.join(REF_DIR, "libref_phase0.so"))
    L.sieve_table_build.argtypes = [C.POINTER(_SieveTable), C.c_int, C.POINTER(_PrimeList)]
    L.sieve_table_build.restype = C.c_int
    L.sieve_apply.argtypes = [C.POINTER(_SieveTable), C.c_longlong, C.c_longlong, C.c_longlong,
                              C.POINTER(C.c_uint32)]
    L.sieve_apply.restype = None
    L.sieve_table_free.argtypes = [C.POINTER(_SieveTable)]
    L.sieve_table_free.restype = None
    small_primes = np.ascontiguousarray(small_primes, dtype=np.uint32)
    pl = _PrimeList(_ptr(small_primes, C.c_uint32), len(small_primes))
    st = _SieveTable()
    if L.sieve_table_build(C.byref(st), 0, C.byref(pl)) != 0:
        raise RuntimeError("sieve_table_build failed")
    out = np.zeros((len(abc), 313), dtype=np.uint32)
    for i, (a, b, c) in enumerate(abc):
        L.sieve_apply(C.byref(st), a, b, c, _ptr(out[i], C.c_uint32))
    L.sieve_table_free(C.byref(st))
    return out


def ref_miller_rabin_test(a: int, b: int, c: int, k: int, j: int) -> int:
    """The reference's own miller_rabin_test (GMP BPSW on N, then rev(N))."""
    global _ref_mr
    if _ref_mr is None:
        _ref_mr = C.CDLL(os.path.join(REF_DIR, "libref_mr.so"))
        _ref_mr.miller_rabin_test.argtypes = [C.c_longlong, C.c_longlong, C.c_longlong,
                                              C.c_int, C.c_int, C.c_void_p]
        _ref_mr.miller_rabin_test.restype = C.c_int
    return _ref_mr.miller_rabin_test(a, b, c, k, j, None)


# -------------------------------------------------------------------- MR ----

def int_to_limbs(x: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint16)
    raw = x.to_bytes(2 * n, "little")
    out[:] = np.frombuffer(raw, dtype="<u2")
    return out


def limbs_to_int(l: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(l, dtype="<u2").tobytes(), "little")


def build_candidate(a: int, b: int, c: int, k: int, j: int, rev: bool) -> int:
    cap = (int(a * 3.3219280948873626) + 64) // 16 + 4
    buf = np.zeros(cap, dtype=np.uint16)
    n = lib().oracle_build_candidate(a, b, c, k, j, int(bool(rev)), _ptr(buf, C.c_uint16), cap)
    if n < 0:
        raise ValueError("bad candidate")
    return limbs_to_int(buf[:n])


def strong_residue(N: int, base: int = 2):
    """(s, base^d mod N) with N - 1 = 2^s d, via mpz_powm."""
    n = (N.bit_length() + 15) // 16
    nl = int_to_limbs(N, n)
    res = np.zeros(n, dtype=np.uint16)
    s = lib().oracle_strong_residue(_ptr(nl, C.c_uint16), n, base, _ptr(res, C.c_uint16), n)
    if s < 0:
        raise ValueError("bad modulus")
    return s, limbs_to_int(res)


def strong_test(N: int, base: int = 2) -> int:
    n = (N.bit_length() + 15) // 16
    nl = int_to_limbs(N, n)
    return lib().oracle_strong_test(_ptr(nl, C.c_uint16), n, base)


def probab_prime(N: int, reps: int = 5) -> int:
    n = (N.bit_length() + 15) // 16
    nl = int_to_limbs(N, n)
    return lib().oracle_probab_prime(_ptr(nl, C.c_uint16), n, reps)


def nextprime(x: int) -> int:
    n = (x.bit_length() + 15) // 16 + 2
    xl = int_to_limbs(x, n)
    out = np.zeros(n, dtype=np.uint16)
    lib().oracle_nextprime(_ptr(xl, C.c_uint16), n, _ptr(out, C.c_uint16), n)
    return limbs_to_int(out)
