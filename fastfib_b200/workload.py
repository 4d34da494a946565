"""Seeded synthetic workloads of the multiply path.

``uneven_products`` draws a stream of independent products with operand bit
lengths log-uniform between 2^lo and 2^hi bits, the two operands of a pair
sized independently within an aspect ratio of at most ``max_aspect``, limbs
uniform random (the top limb's top bit is not forced, so a length is an upper
bound of the bit length, as in user data).
"""
from __future__ import annotations

import math

import numpy as np


def uneven_sizes(seed: int = 4, count: int = 4096, lo: int = 10, hi: int = 24, max_aspect: int = 16):
    """(bits_a, bits_b) pairs: bits_a = 2^U(lo, hi); bits_b = 2^U over the part
    of [lo, hi] within log2(max_aspect) of log2(bits_a)."""
    rng = np.random.default_rng(seed)
    la = rng.uniform(lo, hi, count)
    span = math.log2(max_aspect)
    lb = rng.uniform(np.maximum(lo, la - span), np.minimum(hi, la + span))
    return [(int(2 ** x), int(2 ** y)) for x, y in zip(la, lb)]


def limbs_of_bits(rng: np.random.Generator, bits: int) -> np.ndarray:
    n = max(1, (bits + 63) // 64)
    a = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
    top = bits - 64 * (n - 1)
    if top < 64:
        a[-1] &= np.uint64((1 << top) - 1)
    a[-1] |= np.uint64(1 << (top - 1))
    return a


def uneven_products(seed: int = 4, count: int = 4096, lo: int = 10, hi: int = 24, max_aspect: int = 16):
    """The operand pairs of one uneven batch, as limb arrays."""
    rng = np.random.default_rng(seed + 1)
    return [(limbs_of_bits(rng, a), limbs_of_bits(rng, b)) for a, b in uneven_sizes(seed, count, lo, hi, max_aspect)]
