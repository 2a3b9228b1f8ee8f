"""Shared pytest configuration.

Markers: ``gpu`` - needs a CUDA device (run with ``-m gpu`` on a B200).
Everything else runs on CPU.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "prime-finder_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running parity case")


_PRIMES = {}


def primes_below(limit: int):
    """Odd primes <= limit from the oracle's sieve (cached per process)."""
    if limit not in _PRIMES:
        import oracle
        _PRIMES[limit] = oracle.primes_below(limit)
    return _PRIMES[limit]


@pytest.fixture(scope="session")
def primes_1e8():
    return primes_below(100_000_000)


@pytest.fixture(scope="session")
def primes_2e6():
    return primes_below(2_000_000)
