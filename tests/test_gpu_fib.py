"""GPU parity of fibonacci(n) (src/fib.c:211) through the device chain:
tests/check.py's 245 n against the reference's fibonacci.py (committed as
hashes), tests/bigcheck.ps1's n list and 10^9 through the reference-generated
fingerprints (bit length, low 64 bits, value mod four 64-bit primes), and
limb-exact agreement with the oracle at sizes it finishes in seconds."""
import hashlib
import json
import os
import random

import numpy as np
import pytest

from oracle import limbs_to_int

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def check_ns(seed=1):
    rng = random.Random(seed)
    ns = list(range(200)) + [rng.randint(200, 3_000_000) for _ in range(40)]
    return ns + [4_999_999, 5_000_000, 2**22 - 1, 2**22, 2**22 + 1]


def fingerprint(limbs, primes):
    x = limbs_to_int(limbs)
    return [x.bit_length(), x & (2**64 - 1)] + [x % p for p in primes]


def test_check_py_list(ff):
    gold = load("fib_hex_sha256.json")["sha256"]
    for n in check_ns(1):
        h = format(limbs_to_int(ff.fibonacci(n)), "x")
        assert hashlib.sha256(h.encode()).hexdigest() == gold[str(n)], n


def test_against_oracle(ff, oracle):
    for n in (2**16 + 1, 123457, 10**6, 3 * 10**6 + 7, 2**23, 10**7 + 1):
        assert np.array_equal(ff.fibonacci(n), oracle.fibonacci(n)), n


@pytest.mark.parametrize("n", [10**6, 10**7, 2 * 10**7, 33554431, 50000001, 64 * 10**6, 77777777, 10**8,
                               128000001, 10**9])
def test_fingerprints(ff, n):
    gold = load("fingerprints.json")
    primes = [int(p) for p in gold["primes"]]
    assert fingerprint(ff.fibonacci(n), primes) == [int(v) for v in gold["fingerprints"][str(n)]]


def test_repeatable(ff, oracle):
    """The chain runs eagerly once, is captured into a CUDA graph on the second
    call and replayed after that: every call gives the oracle's limbs."""
    want = oracle.fibonacci(10**7 + 19)
    for _ in range(4):
        assert np.array_equal(ff.fibonacci(10**7 + 19), want)
    other = oracle.fibonacci(3 * 10**6)
    for _ in range(3):  # a second cached chain next to the first
        assert np.array_equal(ff.fibonacci(3 * 10**6), other)
        assert np.array_equal(ff.fibonacci(10**7 + 19), want)
