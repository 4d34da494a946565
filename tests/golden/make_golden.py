"""Generates the committed golden fixtures under tests/golden/.

Run in the build container, where the reference exists:

    python tests/golden/make_golden.py

Sources (all produced here, none written by hand):
* F(n) in hex for tests/check.py's n list (seed 1): the reference's own
  Python oracle fibonacci.py, stored as sha256 of the hex digits.
* Fingerprints (bit length, low 64 bits, F(n) mod the four 64-bit primes of
  tests/memrun.c:22) for bigcheck.ps1's n list, 10^6..10^9 and 2*10^9: the
  reference built from its sources (oracle/_ref) AND, independently, the
  method of tests/fingerprint.py (fast doubling mod p, Binet with mpmath);
  the script refuses to write unless both agree.
* Decimal digits of F(10^6), F(10^7) and F(10^8) (sha256 and digit count)
  from the reference's big_to_string, each checked against Python's str().
  `--decimal-only` rewrites just that file.
* `--add N` adds F(N)'s fingerprint (reference result, checked the same way)
  to fingerprints.json: F(10^10) was added so (6.1 GB of host memory).
"""
import hashlib
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("FASTFIB_REF", "/root/reference")
sys.path.insert(0, ROOT)
sys.path.insert(0, REF)
sys.set_int_max_str_digits(0)

from oracle import Reference, build, int_to_limbs, limbs_to_int  # noqa: E402

P4 = (18446744073709551557, 18446744073709551533, 9223372036854775783, 4611686018427387847)


def check_ns(seed=1):
    """tests/check.py:17-18"""
    rng = random.Random(seed)
    ns = list(range(200)) + [rng.randint(200, 3_000_000) for _ in range(40)]
    return ns + [4_999_999, 5_000_000, 2**22 - 1, 2**22, 2**22 + 1]


def fib_mod(n, m):
    """tests/fingerprint.py:6-14: (F(k), F(k+1)) mod m by fast doubling."""
    def fd(k):
        if k == 0:
            return 0, 1
        a, b = fd(k >> 1)
        c = a * ((2 * b - a) % m) % m
        d = (a * a + b * b) % m
        return (d, (c + d) % m) if k & 1 else (c, d)
    return fd(n)[0]


def binet_bits(n):
    """tests/fingerprint.py:16-20"""
    from mpmath import floor, log, mp, sqrt
    mp.dps = 60
    phi = (1 + sqrt(5)) / 2
    return int(floor(n * log(phi, 2) - log(sqrt(5), 2))) + 1


def fingerprint_limbs(d):
    import numpy as np
    x = int.from_bytes(np.ascontiguousarray(d, dtype=np.uint64).tobytes(), "little")
    return [x.bit_length(), x & (2**64 - 1)] + [x % p for p in P4]


def add_fingerprint(n):
    """One more fingerprint (the reference's result, checked as in main)
    merged into fingerprints.json."""
    path = os.path.join(HERE, "fingerprints.json")
    with open(path) as f:
        gold = json.load(f)
    d = Reference().fibonacci(n)
    mine = fingerprint_limbs(d)
    del d
    indep = [binet_bits(n), fib_mod(n, 2**64)] + [fib_mod(n, p) for p in P4]
    assert mine == indep, (n, mine, indep)
    gold["fingerprints"][str(n)] = [str(v) for v in mine]
    with open(path, "w") as f:
        json.dump(gold, f, indent=1)
    print("fingerprint", n, "ok", flush=True)


def decimal_golden(ref):
    dec = {}
    for n in (10**6, 10**7, 10**8):
        f = ref.fibonacci(n)
        s = ref.to_string(f)
        assert s == str(limbs_to_int(f)), n
        dec[str(n)] = hashlib.sha256(s.encode()).hexdigest()
        dec[f"digits_{n}"] = len(s)
        print("decimal", n, len(s), flush=True)
    with open(os.path.join(HERE, "decimal_sha256.json"), "w") as f:
        json.dump(dec, f, indent=1)


def main():
    build(with_reference=True)
    if "--decimal-only" in sys.argv:
        decimal_golden(Reference())
        return
    if "--add" in sys.argv:
        add_fingerprint(int(sys.argv[sys.argv.index("--add") + 1]))
        return
    from fibonacci import fibonacci  # the reference's Python oracle (fibonacci.py)
    ref = Reference()

    hexes = {}
    for n in check_ns(1):
        h = format(fibonacci(n), "x")
        got = limbs_to_int(ref.fibonacci(n))
        assert got == fibonacci(n), n
        hexes[str(n)] = hashlib.sha256(h.encode()).hexdigest()

    fps = {}
    for n in (10**6, 10**7, 2 * 10**7, 33554431, 50000001, 64 * 10**6, 77777777, 10**8, 128000001, 10**9,
              2 * 10**9):
        d = ref.fibonacci(n)
        mine = fingerprint_limbs(d)
        indep = [binet_bits(n), fib_mod(n, 2**64)] + [fib_mod(n, p) for p in P4]
        assert mine == indep, (n, mine, indep)
        fps[str(n)] = mine
        print("fingerprint", n, "ok", flush=True)


    with open(os.path.join(HERE, "fib_hex_sha256.json"), "w") as f:
        json.dump({"source": "fibonacci.py (reference) for tests/check.py's n list, seed 1", "sha256": hexes}, f,
                  indent=0)
    with open(os.path.join(HERE, "fingerprints.json"), "w") as f:
        json.dump({"primes": [str(p) for p in P4], "fields": ["bits", "low64", "mod_a", "mod_b", "mod_c", "mod_d"],
                   "fingerprints": {k: [str(v) for v in vals] for k, vals in fps.items()}}, f, indent=1)
    decimal_golden(ref)
    print("written")


if __name__ == "__main__":
    main()
