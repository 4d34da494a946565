"""CPU tests of the synthetic workloads: the uneven product stream keeps its
stated distribution (4096 products, 2^10..2^24 bits, aspect at most 16:1)."""
import math

import numpy as np

from fastfib_b200.workload import limbs_of_bits, uneven_sizes


def test_uneven_sizes():
    s = uneven_sizes(seed=4, count=4096)
    assert len(s) == 4096
    for a, b in s:
        assert 2**10 <= a <= 2**24 and 2**10 <= b <= 2**24
        assert max(a, b) <= 16 * min(a, b) + 1
    la = np.array([math.log2(a) for a, _ in s])
    assert abs(la.mean() - 17) < 0.2  # log-uniform over [10, 24]
    assert uneven_sizes(seed=4, count=4096) == s  # seeded


def test_limbs_of_bits():
    rng = np.random.default_rng(1)
    for bits in (1, 63, 64, 65, 1000, 4096):
        a = limbs_of_bits(rng, bits)
        x = int.from_bytes(a.tobytes(), "little")
        assert x.bit_length() == bits and a.size == (bits + 63) // 64
