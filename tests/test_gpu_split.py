"""GPU parity of the piecewise split multiply (src/mul_split.c:98-187): the
transform cap forced down the way the reference's -DNTT_MAX_LG=10 / 12 / 23
test builds do (tests/test.ps1:29, 39), so products past the cap are cut into
pieces transformed once and combined pointwise; plans match the oracle's
restatement of the split's width and piece-length choice, products match
exact integers limb for limb, and F(10^9) with the cap at 2^23 (the split
for its last squarings and final product) matches its fingerprint."""
import json
import os
import random

import numpy as np
import pytest

from oracle import int_to_limbs, limbs_to_int

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture
def capped(ff, oracle):
    def set_cap(lg):
        ff.ntt_init(1 << 24)
        oracle.ntt_init(1 << 24)
        ff.set_max_lg(lg)
        oracle.set_max_lg(lg)
    yield set_cap
    ff.set_max_lg(25)
    oracle.set_max_lg(25)
    ff.ntt_init(1 << 24)
    oracle.ntt_init(1 << 24)


@pytest.mark.parametrize("lg", [10, 12])
def test_split_products(ff, oracle, capped, lg):
    capped(lg)
    rng = random.Random(lg)
    splits = 0
    for na, nb in ((600, 600), (3000, 1000), (5000, 5000), (12000, 700), (40000, 33000)):
        x, y = rng.getrandbits(64 * na) | 1 << (64 * na - 1), rng.getrandbits(64 * nb) | 1
        pf = ff.plan(x.bit_length(), y.bit_length(), False)
        po = oracle.plan(x.bit_length(), y.bit_length(), False)
        assert pf["split"] == po.split
        assert (pf["width"], pf["L"], pf["ka"], pf["kb"], pf["Lbig"]) == (po.width, po.L, po.ka, po.kb, po.Lbig)
        splits += pf["split"]
        assert limbs_to_int(ff.big_mul_ntt(int_to_limbs(x), int_to_limbs(y))) == x * y
        assert limbs_to_int(ff.big_mul_ntt(int_to_limbs(x))) == x * x
    assert splits >= 4


def test_split_all_ones(ff, capped):
    """The CRT bound's worst case through the split (tests/bound.c's operands)."""
    capped(12)
    for nl in (3000, 20000):
        N = 64 * nl
        a = np.full(nl, 0xFFFFFFFFFFFFFFFF, dtype=np.uint64)
        assert limbs_to_int(ff.big_mul_ntt(a)) == (1 << (2 * N)) - (1 << (N + 1)) + 1


def test_fib_with_split(ff, oracle, capped):
    capped(12)
    for n in (10**6 + 3, 5 * 10**6):
        assert np.array_equal(ff.fibonacci(n), oracle.fibonacci(n))


def test_f1e9_split_cap23(ff, capped):
    """F(10^9) with NTT_MAX_LG = 23: its last squarings and final product split."""
    capped(23)
    with open(os.path.join(GOLD, "fingerprints.json")) as f:
        gold = json.load(f)
    x = limbs_to_int(ff.fibonacci(10**9))
    fp = [x.bit_length(), x & (2**64 - 1)] + [x % int(p) for p in gold["primes"]]
    assert [str(v) for v in fp] == gold["fingerprints"]["1000000000"]


def test_f1e10(ff):
    """F(10^10) (6.9 * 10^9 bits): the split at pieces of 2^25 past 32-bit
    bit positions, against the reference-generated fingerprint; the 868 MB
    result is fingerprinted on the device (its kernel is checked against
    Python integers in test_gpu_fingerprint.py)."""
    with open(os.path.join(GOLD, "fingerprints.json")) as f:
        gold = json.load(f)
    r = ff.fibonacci(10**10)
    assert ff.fingerprint(r) == [int(v) for v in gold["fingerprints"]["10000000000"]]


@pytest.mark.parametrize("lg", [4, 5, 6, 7, 8, 9])
def test_split_tiny_pieces(ff, oracle, capped, lg):
    """Transform caps of 2^4..2^9 (NTT_MAX_LG builds that low) split into
    pieces as short as 16 coefficients: rows of 4 words, columns of 4."""
    capped(lg)
    rng = random.Random(100 + lg)
    splits = 0
    for na, nb in ((40, 40), (100, 37), (300, 300)):
        x, y = rng.getrandbits(64 * na), rng.getrandbits(64 * nb)
        splits += ff.plan(64 * na, 64 * nb)["split"]
        assert limbs_to_int(ff.big_mul_ntt(int_to_limbs(x), int_to_limbs(y))) == x * y, (lg, na, nb)
        assert limbs_to_int(ff.big_mul_ntt(int_to_limbs(x))) == x * x, (lg, na)
    assert splits >= 1
