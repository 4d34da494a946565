"""GPU parity of the device decimal conversion (big_to_string,
src/decimal.c:229-281, level by level with batched Barrett products): the
digits of F(10^6), F(10^7) and F(10^8) against the reference's own output
(sha256 and digit count, tests/golden/decimal_sha256.json), and numbers at
the edges of the divide and conquer -- one below / at / above powers of ten
at every split size, all-ones, sparse pieces of zeros -- against Python's
str().  Each case checks that the device path ran (done = True)."""
import hashlib
import json
import os
import random

import numpy as np
import pytest

from oracle import int_to_limbs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "decimal_sha256.json")


def device_digits(ff, x):
    s, done = ff.to_decimal(int_to_limbs(x) if isinstance(x, int) else x)
    assert done, "the device path declined: " + ff.lib().ffg_last_error().decode()
    return s


@pytest.mark.parametrize("n", [10**6, 10**7, 10**8])
def test_fibonacci_digits(ff, n):
    with open(GOLD) as f:
        gold = json.load(f)
    s = device_digits(ff, ff.fibonacci(n))
    assert len(s) == gold[f"digits_{n}"]
    assert hashlib.sha256(s.encode()).hexdigest() == gold[str(n)]


def test_powers_of_ten_edges(ff):
    for lg in range(9, 13):
        for k in ((19 << lg) - 1, 19 << lg, (19 << lg) + 1, (38 << lg) - 1):
            for d in (-1, 0, 1):
                x = 10**k + d
                assert device_digits(ff, x) == str(x), (k, d)


def test_all_ones_and_sparse(ff):
    rng = random.Random(3)
    cases = [2**b - 1 for b in (20000, 65536, 131071, 500000)]
    cases += [10**60000 * rng.getrandbits(64) + rng.getrandbits(64) for _ in range(3)]  # zero pieces inside
    cases += [rng.getrandbits(rng.randint(16384, 400000)) for _ in range(10)]
    for x in cases:
        assert device_digits(ff, x) == str(x)


def test_big_to_string_takes_the_device_path(ff):
    x = random.Random(4).getrandbits(300000)
    assert ff.big_to_string(int_to_limbs(x)) == str(x)


def test_device_pointer_entry(ff):
    torch = pytest.importorskip("torch")
    x = random.Random(5).getrandbits(250000)
    a = int_to_limbs(x)
    t = torch.from_numpy(a.view(np.int64)).cuda()
    s, done = ff.to_decimal(None, device_ptr=t.data_ptr(), n=a.size)
    assert done and s == str(x)


def test_after_other_work(ff):
    """The arena is reused across calls: a conversion after a large batch of
    products (its buffers full of other data) must still be exact, and every
    ticket of the in-launch carry settle must be back at zero."""
    from fastfib_b200.workload import uneven_products
    with open(GOLD) as f:
        gold = json.load(f)
    x = ff.fibonacci(10**7)
    assert hashlib.sha256(device_digits(ff, x).encode()).hexdigest() == gold["10000000"]
    ff.mul_batch(uneven_products(seed=9, count=1500, lo=12, hi=23), "plain")
    for _ in range(2):
        assert hashlib.sha256(device_digits(ff, x).encode()).hexdigest() == gold["10000000"]
    assert ff.tickets_in_use() == 0


def test_streamed_digits(ff):
    """ffg_to_decimal_stream (the command line's streamed output): the slices
    joined are the reference's digits of F(10^7) (hash), there is more than
    one slice, and numbers whose top slices are all leading zeros stream
    exactly str()'s digits."""
    with open(GOLD) as f:
        gold = json.load(f)
    pieces, done = ff.to_decimal_stream(ff.fibonacci(10**7))
    assert done and len(pieces) > 1
    s = "".join(pieces)
    assert len(s) == gold[f"digits_{10**7}"]
    assert hashlib.sha256(s.encode()).hexdigest() == gold[str(10**7)]
    for x in (10**(19 << 9) + 12345, (1 << 60000) + 1, 10**(38 << 8) - 1):
        pieces, done = ff.to_decimal_stream(int_to_limbs(x))
        assert done
        assert "".join(pieces) == str(x)
    assert ff.to_decimal_stream(int_to_limbs(12345)) == ([], False)  # below 10^2432: declined
