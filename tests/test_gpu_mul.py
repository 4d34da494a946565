"""GPU parity of the NTT multiply (big_mul_ntt, src/mul_ntt.c:97) against the
oracle and exact Python integers: random, all-ones and sparse operands in the
generator of tests/nttfuzz.c (xorshift64, seed 88172645463325252), squares
and distinct products, across the one-CTA and four-step kernels and both
length families (2^k and 3 * 2^k), plus the all-ones CRT-bound cases of
tests/bound.c.  Bit-exact: every limb must match."""
import numpy as np
import pytest

from oracle import int_to_limbs, limbs_to_int

pytestmark = pytest.mark.gpu


class XorShift:
    """tests/nttfuzz.c:10-18"""

    def __init__(self, seed=88172645463325252):
        self.s = seed

    def __call__(self):
        s = self.s
        s ^= (s << 13) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 7
        s ^= (s << 17) & 0xFFFFFFFFFFFFFFFF
        self.s = s
        return s


def make(rng, n, kind):
    """tests/nttfuzz.c:23-30: random, all ones, or sparse; top bit set."""
    d = np.empty(n, dtype=np.uint64)
    for i in range(n):
        if kind == 0:
            d[i] = rng()
        elif kind == 1:
            d[i] = 0xFFFFFFFFFFFFFFFF
        else:
            d[i] = rng() if rng() % 7 == 0 else 0
    d[n - 1] |= np.uint64(1 << 63)
    return d


@pytest.fixture(scope="module", autouse=True)
def _init(ff):
    ff.init(1 << 22)


def check(ff, a, b=None):
    got = ff.mul(a) if b is None else ff.mul(a, b)
    A = limbs_to_int(a)
    want = A * A if b is None else A * limbs_to_int(b)
    assert limbs_to_int(got) == want
    assert got.size == max(1, (want.bit_length() + 63) // 64)


def test_fuzz_small(ff):
    rng = XorShift()
    for t in range(150):
        na = 1 + rng() % 2000
        nb = 1 + rng() % na if rng() % 3 == 0 else na
        a, b = make(rng, na, rng() % 3), make(rng, nb, rng() % 3)
        if rng() % 3 == 0:
            check(ff, a)
        else:
            check(ff, a, b)


def test_fuzz_large(ff):
    rng = XorShift(12345)
    for t in range(12):
        na = 1 + rng() % 60000
        nb = 1 + rng() % na if rng() % 3 == 0 else na
        a, b = make(rng, na, rng() % 3), make(rng, nb, rng() % 3)
        check(ff, a) if t % 3 == 0 else check(ff, a, b)


@pytest.mark.parametrize("nlimbs", [200, 1000, 5000, 20000, 100000, 300000])
def test_all_ones_square(ff, nlimbs):
    """tests/bound.c: (2^N - 1)^2 in closed form, every coefficient at its maximum."""
    N = 64 * nlimbs
    a = np.full(nlimbs, 0xFFFFFFFFFFFFFFFF, dtype=np.uint64)
    got = limbs_to_int(ff.mul(a))
    assert got == (1 << (2 * N)) - (1 << (N + 1)) + 1


def test_lengths_both_families(ff, oracle):
    """Sizes whose plan lands on 2^k and on 3 * 2^k, one-CTA and four-step."""
    oracle.ntt_init(1 << 22)
    rng = np.random.default_rng(7)
    seen = set()
    for n in [60, 100, 130, 190, 260, 400, 700, 1000, 1500, 2100, 3000, 4200, 6000, 9000, 13000, 20000,
              33000, 50000, 70000, 140000, 270000]:
        a = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
        a[-1] |= np.uint64(1 << 63)
        pl = ff.plan(64 * n, 64 * n, True)
        seen.add((pl["r3"], pl["kernel"]))
        po = oracle.plan(64 * n, 64 * n, True)
        assert (pl["width"], pl["L"]) == (po.width, po.L)
        check(ff, a)
        b = rng.integers(0, 2**64, n // 2 + 1, dtype=np.uint64)
        b[-1] |= np.uint64(1)
        check(ff, a, b)
    assert seen == {(0, 0), (1, 0), (0, 1), (1, 1)}


def test_edge_operands(ff):
    one = np.array([1], dtype=np.uint64)
    zero = np.array([0], dtype=np.uint64)
    big = np.full(500, 0xFFFFFFFFFFFFFFFF, dtype=np.uint64)
    assert limbs_to_int(ff.mul(big, zero)) == 0
    assert limbs_to_int(ff.mul(big, one)) == limbs_to_int(big)
    padded = np.concatenate([big, np.zeros(7, dtype=np.uint64)])  # leading zero limbs
    assert limbs_to_int(ff.mul(padded, big)) == limbs_to_int(big) ** 2
