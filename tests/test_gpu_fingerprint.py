"""GPU parity of the device fingerprint (the check format of the reference's
tests/memrun.c:19-27: bit length, low 64 bits, value mod four 64-bit primes)
against Python integers on seeded limbs: empty, one limb, zero top limbs,
all zeros, lengths that leave threads empty or ragged, a top limb of every
bit length; and against the reference-generated fingerprints of F(n) for n
where the result is taken straight from the device chain's output."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
P4 = (18446744073709551557, 18446744073709551533, 9223372036854775783, 4611686018427387847)


def expect(limbs):
    x = int.from_bytes(np.ascontiguousarray(limbs, dtype=np.uint64).tobytes(), "little")
    return [x.bit_length(), x & (2**64 - 1)] + [x % p for p in P4]


def test_primes_exported(ff):
    assert tuple(ff.FP_PRIMES) == P4


@pytest.mark.parametrize("n", [0, 1, 2, 3, 255, 256, 257, 151551, 151552, 151553, 592 * 256 * 3 + 7, 1 << 20,
                               10**6 + 3])
def test_random(ff, n):
    rng = np.random.default_rng(n + 5)
    a = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    assert ff.fingerprint(a) == expect(a), n


def test_zero_tops_and_zeros(ff):
    rng = np.random.default_rng(9)
    a = rng.integers(0, 2**64, size=100_003, dtype=np.uint64)
    a[50_000:] = 0
    assert ff.fingerprint(a) == expect(a)
    z = np.zeros(70_001, np.uint64)
    assert ff.fingerprint(z) == [0, 0, 0, 0, 0, 0]
    all_ones = np.full(9_999, 2**64 - 1, np.uint64)
    assert ff.fingerprint(all_ones) == expect(all_ones)


def test_top_bits(ff):
    rng = np.random.default_rng(3)
    base = rng.integers(0, 2**64, size=40_000, dtype=np.uint64)
    for b in range(64):
        a = base.copy()
        a[-1] = np.uint64(1) << np.uint64(b)
        assert ff.fingerprint(a) == expect(a), b


def test_device_pointer(ff):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(21)
    a = rng.integers(0, 2**64, size=3_000_001, dtype=np.uint64)
    t = torch.from_numpy(a.view(np.int64)).to("cuda:0")
    assert ff.fingerprint(device_ptr=t.data_ptr(), n=t.numel()) == expect(a)
    # a view starting mid-buffer
    assert ff.fingerprint(device_ptr=t[1000:].data_ptr(), n=t.numel() - 1000) == expect(a[1000:])


@pytest.mark.parametrize("n", [10**8, 10**9])
def test_fib_golden(ff, n):
    with open(os.path.join(GOLD, "fingerprints.json")) as f:
        gold = json.load(f)
    assert ff.fingerprint(ff.fibonacci(n)) == [int(v) for v in gold["fingerprints"][str(n)]]
