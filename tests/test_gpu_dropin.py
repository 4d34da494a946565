"""Drop-in check: the reference's own test harnesses, compiled unmodified
against this library's C surface (`make -C oracle dropin`: each harness's
`#include "../fastfib.c"` finds oracle/dropin/fastfib.c, which includes
include/fastfib.h, and the binary links libfastfib_b200.so), run on the GPU:

* tests/hexfib.c   -- F(n) in hex for tests/check.py's n list, against the
                      reference's fibonacci.py (committed as hashes);
* tests/nttfuzz.c  -- 601 big_mul_ntt products against big_mul with the NTT
                      hidden (g_ntt_max_L = 0: Karatsuba / Toom-3);
* tests/bound.c    -- the CRT-bound all-ones squares and products up to 4M
                      limbs against their closed forms;
* tests/dectest.c  -- big_to_string on tests/dectest.py's number classes
                      (restated here, Python's str standing in for gmpy2).

The binaries are built where the reference's sources are (the build step)
and travel with the repository; without them the tests skip."""
import hashlib
import json
import os
import random
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROP = os.path.join(ROOT, "oracle", "_ref", "dropin")


def harness(name):
    exe = os.path.join(DROP, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (make -C oracle dropin needs the reference's sources)")
    return exe


def check_ns(seed=1):
    """tests/check.py:17-18"""
    rng = random.Random(seed)
    ns = list(range(200)) + [rng.randint(200, 3_000_000) for _ in range(40)]
    return ns + [4_999_999, 5_000_000, 2**22 - 1, 2**22, 2**22 + 1]


def test_hexfib(ff):
    with open(os.path.join(ROOT, "tests", "golden", "fib_hex_sha256.json")) as f:
        gold = json.load(f)["sha256"]
    ns = check_ns(1)
    r = subprocess.run([harness("hexfib"), *map(str, ns)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.split("\n")
    for n, line in zip(ns, lines):
        assert hashlib.sha256(line.encode()).hexdigest() == gold[str(n)], n
    assert len(lines) >= len(ns)


def test_nttfuzz(ff):
    r = subprocess.run([harness("nttfuzz")], capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, (r.stdout + r.stderr)[-2000:]
    assert "601 trials, 0 failures" in r.stdout


def test_bound(ff):
    r = subprocess.run([harness("bound")], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (r.stdout + r.stderr)[-2000:]
    assert "9 products, 0 failures" in r.stdout
    assert r.stdout.count(": ok") == 9


def _fib(n):
    a, b = 0, 1  # (F(k), F(k+1)) by fast doubling
    for bit in bin(n)[2:]:
        c = a * (2 * b - a)
        d = a * a + b * b
        a, b = (d, c + d) if bit == "1" else (c, d)
    return a


def dectest_numbers(seed=1):
    """tests/dectest.py:6-21 (gmpy2.fib replaced by fast doubling)."""
    rng = random.Random(seed)
    nums = [0, 1, 9, 10, 2**64 - 1, 2**64, 10**19 - 1, 10**19, 10**19 + 1]
    for i in range(0, 12):
        for k in (19 << i, (19 << i) + 1, (19 << i) - 1, (38 << i), (38 << i) - 1):
            for d in (-1, 0, 1):
                nums.append(10**k + d)
    for b in (64, 128, 1000, 2047, 2048, 2049, 4096, 10000, 65536, 200000):
        nums += [2**b - 1, 2**b, 2**b + 1]
    for _ in range(300):
        bits = int(2 ** rng.uniform(1, 20))
        x = rng.getrandbits(bits)
        if rng.random() < 0.3:
            x = x * 10**rng.randint(1, 5000) + rng.getrandbits(rng.randint(1, 64))
        nums.append(x)
    for n in (1000, 100000, 1000000, 3000000):
        nums.append(_fib(n))
    return nums


def test_dectest(ff):
    nums = dectest_numbers(1)
    inp = "".join(format(x, "x") + "\n" for x in nums)
    r = subprocess.run([harness("dectest")], input=inp, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    out = r.stdout.split("\n")
    bad = [i for i, x in enumerate(nums) if out[i] != str(x)]
    assert not bad, f"{len(nums)} numbers, {len(bad)} mismatches (first: index {bad[0]})"
