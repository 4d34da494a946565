"""CPU tests: the oracle (our scalar C restatement) pinned against the
reference's own known answers and against the reference built from its
sources.  No GPU needed."""
import hashlib
import json
import os
import random

import numpy as np
import pytest

from oracle import int_to_limbs, limbs_to_int

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def check_ns(seed=1):
    """tests/check.py:17-18"""
    rng = random.Random(seed)
    ns = list(range(200)) + [rng.randint(200, 3_000_000) for _ in range(40)]
    return ns + [4_999_999, 5_000_000, 2**22 - 1, 2**22, 2**22 + 1]


def test_fib_hex_against_fibonacci_py(oracle):
    """check.py: F(n) in hex for 245 n against the reference's fibonacci.py."""
    gold = load("fib_hex_sha256.json")["sha256"]
    ns = check_ns(1)
    assert len(gold) == len(ns)
    for n in ns:
        h = format(limbs_to_int(oracle.fibonacci(n)), "x")
        assert hashlib.sha256(h.encode()).hexdigest() == gold[str(n)], n


@pytest.mark.parametrize("n", [10**6, 10**7, 2 * 10**7, 33554431])
def test_fingerprints(oracle, n):
    """memrun.c / fingerprint.py fingerprints, generated by the reference and
    checked there against the independent Binet / mod-p computation."""
    fp = [int(v) for v in load("fingerprints.json")["fingerprints"][str(n)]]
    assert list(oracle.fingerprint(oracle.fibonacci(n))) == fp


def test_cli_known_values(oracle):
    """cli.ps1:15-16: F(93) is the last Fibonacci number below 2^64."""
    assert limbs_to_int(oracle.fibonacci(93)) == 12200160415121876738
    assert limbs_to_int(oracle.fibonacci(94)) == 19740274219868223167


def test_decimal_golden(oracle):
    gold = load("decimal_sha256.json")
    s = oracle.to_string(oracle.fibonacci(10**6))
    assert len(s) == gold["digits_1000000"] == 208988
    assert hashlib.sha256(s.encode()).hexdigest() == gold["1000000"]


def dectest_numbers(seed=1, random_count=60, max_split=9):
    """tests/dectest.py:7-21 number classes (a reduced random count)."""
    rng = random.Random(seed)
    nums = [0, 1, 9, 10, 2**64 - 1, 2**64, 10**19 - 1, 10**19, 10**19 + 1]
    for i in range(0, max_split):
        for k in (19 << i, (19 << i) + 1, (19 << i) - 1, (38 << i), (38 << i) - 1):
            for d in (-1, 0, 1):
                nums.append(10**k + d)
    for b in (64, 128, 1000, 2047, 2048, 2049, 4096, 10000, 65536, 200000):
        nums += [2**b - 1, 2**b, 2**b + 1]
    for _ in range(random_count):
        bits = int(2 ** rng.uniform(1, 18))
        x = rng.getrandbits(bits)
        if rng.random() < 0.3:
            x = x * 10 ** rng.randint(1, 2000) + rng.getrandbits(rng.randint(1, 64))
        nums.append(x)
    return nums


def test_decimal_classes(oracle):
    for x in dectest_numbers():
        assert oracle.to_string(int_to_limbs(x)) == str(x)


class XorShift:
    def __init__(self, seed=88172645463325252):
        self.s = seed

    def __call__(self):
        s = self.s
        s ^= (s << 13) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 7
        s ^= (s << 17) & 0xFFFFFFFFFFFFFFFF
        self.s = s
        return s


def test_nttfuzz_generator(oracle):
    """tests/nttfuzz.c: products through the NTT path against exact integers."""
    oracle.ntt_init(1 << 18)
    rng = XorShift()
    for t in range(120):
        na = 1 + rng() % 2000
        nb = 1 + rng() % na if rng() % 3 == 0 else na
        ka = rng() % 3  # the call order of tests/nttfuzz.c:45-49
        A = [rng() if ka == 0 else (2**64 - 1 if ka == 1 else (rng() if rng() % 7 == 0 else 0)) for _ in range(na)]
        kb = rng() % 3
        B = [rng() if kb == 0 else (2**64 - 1 if kb == 1 else (rng() if rng() % 7 == 0 else 0)) for _ in range(nb)]
        A[-1] |= 1 << 63
        B[-1] |= 1 << 63
        a_, b_ = np.array(A, dtype=np.uint64), np.array(B, dtype=np.uint64)
        x, y = limbs_to_int(a_), limbs_to_int(b_)
        if rng() % 3 == 0:
            assert limbs_to_int(oracle.mul_ntt(a_)) == x * x
        else:
            assert limbs_to_int(oracle.mul_ntt(a_, b_)) == x * y


@pytest.mark.parametrize("bits", [64 * 1000, 64 * 100000 + 17])
def test_bound_all_ones(oracle, bits):
    """tests/bound.c:30: (2^N - 1)^2 = 2^2N - 2^(N+1) + 1 at every coefficient's maximum."""
    oracle.ntt_init(8000000)
    a = int_to_limbs((1 << bits) - 1)
    assert limbs_to_int(oracle.mul_ntt(a)) == (1 << (2 * bits)) - (1 << (bits + 1)) + 1


def test_split_forced(oracle):
    """The split multiply forced from small sizes (test.ps1's -DNTT_MAX_LG=10 idea)."""
    saved = oracle.ntt_max_L()
    try:
        oracle.set_ntt_max_L(1 << 10)
        rng = random.Random(3)
        for na, nb in ((5000, 3000), (4096, 4096), (700, 9000)):
            x, y = rng.getrandbits(64 * na), rng.getrandbits(64 * nb)
            pl = oracle.plan(x.bit_length(), y.bit_length())
            assert pl.split == 1
            assert limbs_to_int(oracle.mul_ntt(int_to_limbs(x), int_to_limbs(y))) == x * y
            assert limbs_to_int(oracle.mul_ntt(int_to_limbs(x))) == x * x
    finally:
        oracle.set_ntt_max_L(saved)


def test_plan_matches_reference_choice(oracle):
    """The width / length choice of big_mul_ntt at the microbench sizes
    (2^14, 2^17, 2^20, 2^22 limbs squared -> L = 2^16, 2^19, 2^22, 2^24 at b = 32, as the
    reference build picks them)."""
    oracle.ntt_init(1 << 24)
    for lg_limbs, lg_L in ((14, 16), (17, 19), (20, 22), (22, 24)):
        bits = 64 << lg_limbs
        pl = oracle.plan(bits, bits, True)
        assert (pl.width, pl.L, pl.split) == (32, 1 << lg_L, 0)


def test_oracle_against_reference(oracle, reference):
    """Same products / F(n) / digits as the unmodified reference."""
    reference.ntt_init(1 << 18)
    rng = np.random.default_rng(11)
    for n in (250, 1300, 7000, 40000):
        a = rng.integers(0, 2**64, n, dtype=np.uint64)
        b = rng.integers(0, 2**64, n // 3 + 1, dtype=np.uint64)
        assert np.array_equal(oracle.mul(a, b), reference.mul(a, b))
        assert np.array_equal(oracle.mul(a), reference.mul(a))
    for n in (1000, 99999, 1234567):
        f = oracle.fibonacci(n)
        assert np.array_equal(f, reference.fibonacci(n))
        if n < 200000:
            assert oracle.to_string(f) == reference.to_string(f)


@pytest.mark.parametrize("lg", [4, 6, 8])
def test_split_tiny_caps(oracle, lg):
    """The split multiply under transform caps of 2^4..2^8 (pieces as short as
    16 coefficients), as the GPU's test_split_tiny_pieces runs it."""
    saved = oracle.ntt_max_L()
    try:
        oracle.set_ntt_max_L(1 << lg)
        rng = random.Random(200 + lg)
        for na, nb in ((40, 40), (100, 37), (300, 300)):
            x, y = rng.getrandbits(64 * na), rng.getrandbits(64 * nb)
            assert limbs_to_int(oracle.mul_ntt(int_to_limbs(x), int_to_limbs(y))) == x * y, (lg, na, nb)
            assert limbs_to_int(oracle.mul_ntt(int_to_limbs(x))) == x * x, (lg, na)
    finally:
        oracle.set_ntt_max_L(saved)


@pytest.mark.parametrize("square", [False, True])
def test_residues_are_the_digit_convolution(oracle, square):
    """One prime's share of a prime-sharded product (fo_residues) is the plain
    convolution of the operands' width-w digits modulo that prime, word for
    word, zero past the product's coefficients; the three shares' CRT
    (fo_crt_residues) is the product."""
    P = (2113929217, 2013265921, 1811939329)
    rng = np.random.default_rng(11)
    a = rng.integers(0, 2**64, 37, dtype=np.uint64)
    b = a if square else rng.integers(0, 2**64, 29, dtype=np.uint64)
    x, y = limbs_to_int(a), limbs_to_int(b)
    for w, L in ((32, 256), (35, 192)):
        ca, cb = -(-x.bit_length() // w), -(-y.bit_length() // w)
        da = [(x >> (w * i)) & ((1 << w) - 1) for i in range(ca)]
        db = [(y >> (w * i)) & ((1 << w) - 1) for i in range(cb)]
        conv = [0] * (ca + cb - 1)
        for i, u in enumerate(da):
            for j, v in enumerate(db):
                conv[i + j] += u * v
        ys = []
        for k, p in enumerate(P):
            got = oracle.residues(a, b, w, L, k, square)
            assert [int(v) for v in got[:len(conv)]] == [c % p for c in conv], (w, k)
            assert not got[len(conv):].any()
            ys.append(got)
        prod = oracle.crt_residues(np.stack(ys), L, len(conv), w, a.size + b.size + 1)
        assert limbs_to_int(prod) == x * y
    with pytest.raises(ValueError):  # a length that does not hold the product
        oracle.residues(a, b, 32, 64, 0, square)
