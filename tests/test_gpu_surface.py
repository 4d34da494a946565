"""The reference's C surface served by the GPU layer: the threshold dispatch
(big_mul / big_sqr, src/mul_basic.c:64-132) with the NTT on the device, the
transform cap g_ntt_max_L (0 hides the NTT, as tests/nttfuzz.c:33-39 does),
Toom-3, and big_to_string (src/decimal.c:229) on tests/dectest.py's number
classes against Python's str()."""
import random

import numpy as np
import pytest

from oracle import int_to_limbs, limbs_to_int

pytestmark = pytest.mark.gpu


def test_dispatch_all_paths(ff):
    ff.ntt_init(1 << 18)
    rng = random.Random(5)
    for na, nb in ((3, 5), (64, 64), (65, 130), (150, 199), (200, 200), (250, 1000), (1499, 1600), (4000, 3000),
                   (30000, 20)):
        x, y = rng.getrandbits(64 * na), rng.getrandbits(64 * nb)
        assert limbs_to_int(ff.big_mul(int_to_limbs(x), int_to_limbs(y))) == x * y
        assert limbs_to_int(ff.big_sqr(int_to_limbs(x))) == x * x


def test_toom3_when_the_ntt_is_hidden(ff):
    saved = ff.g_ntt_max_L()
    try:
        ff.set_g_ntt_max_L(0)
        rng = random.Random(6)
        for na, nb in ((1600, 1600), (5000, 2000)):
            x, y = rng.getrandbits(64 * na), rng.getrandbits(64 * nb)
            assert limbs_to_int(ff.big_mul(int_to_limbs(x), int_to_limbs(y))) == x * y
            assert limbs_to_int(ff.big_sqr(int_to_limbs(x))) == x * x
    finally:
        ff.set_g_ntt_max_L(saved)


def test_big_mul_ntt_square_by_pointer(ff):
    x = random.Random(7).getrandbits(64 * 3000)
    assert limbs_to_int(ff.big_mul_ntt(int_to_limbs(x))) == x * x


def dectest_numbers(seed=1):
    rng = random.Random(seed)
    nums = [0, 1, 9, 10, 2**64 - 1, 2**64, 10**19 - 1, 10**19, 10**19 + 1]
    for i in range(0, 11):
        for k in (19 << i, (19 << i) + 1, (19 << i) - 1, (38 << i), (38 << i) - 1):
            for d in (-1, 0, 1):
                nums.append(10**k + d)
    for b in (64, 128, 1000, 2047, 2048, 2049, 4096, 10000, 65536, 200000):
        nums += [2**b - 1, 2**b, 2**b + 1]
    for _ in range(120):
        bits = int(2 ** rng.uniform(1, 20))
        x = rng.getrandbits(bits)
        if rng.random() < 0.3:
            x = x * 10 ** rng.randint(1, 5000) + rng.getrandbits(rng.randint(1, 64))
        nums.append(x)
    return nums


def test_decimal_classes(ff):
    for x in dectest_numbers():
        assert ff.big_to_string(int_to_limbs(x)) == str(x)


def test_decimal_of_fibonacci(ff, oracle):
    f = ff.fibonacci(10**6)
    assert ff.big_to_string(f) == oracle.to_string(f)
