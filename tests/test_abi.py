"""CPU tests of the boundary: the library builds, loads without a GPU, and
exports every function declared in include/*.h; the plan logic is host-only
and checked against the oracle's restatement of big_mul_ntt's choice."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for fn in os.listdir(INC):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INC, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"typedef[^;]*;", "", text)  # function-pointer types declare no symbol
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.add(name)
    return names


def test_header_has_the_reference_surface():
    names = declared_functions()
    for n in ("big_mul", "big_sqr", "big_mul_ntt", "fibonacci", "big_to_string", "ntt_init", "big_free",
              "ffg_init", "ffg_mul_host", "ffg_mul_device", "ffg_fib_chain", "ffg_plan_select", "ffg_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(ff):
    lib = ff.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing
    ctypes.c_size_t.in_dll(lib, "g_ntt_max_L")  # the reference's global, exported too


def test_plan_select_without_gpu(ff, oracle):
    """Plans need no device: they mirror big_mul_ntt's width / length choice."""
    oracle.ntt_init(1 << 22)
    ff.lib().ffg_set_ntt_max_L(oracle.ntt_max_L())
    for bits_a, bits_b in ((6400, 6400), (64 * 1356, 64 * 1356), (64 * 5424, 64 * 5424), (64 * 10000, 64 * 333),
                           (64 * 542377, 64 * 542377), (64 * 271189, 64 * 271189), (100, 64 * 2000)):
        for sq in ((True, False) if bits_a == bits_b else (False,)):
            p = ff.plan(bits_a, bits_b, sq)
            o = oracle.plan(bits_a, bits_b, sq)
            assert (p["width"], p["L"], p["lg"], p["r3"], p["conv"]) == (o.width, o.L, o.lg, o.r3, o.conv)


def test_gpu_calls_fail_loudly_without_gpu(ff):
    import numpy as np
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(ff.FfgError):
        ff.mul(np.ones(300, dtype=np.uint64))


def test_plan_select_sweep(ff, oracle):
    """The width / length / split choice of big_mul_ntt (src/mul_ntt.c:97-118,
    src/mul_split.c:150-177) on 1500 seeded shapes, squares and distinct,
    log-uniform 2^6..2^28 bits, under transform caps 2^10, 2^16, 2^22 and
    2^25: every field the oracle restatement gives, the split's included."""
    import math
    import random
    rng = random.Random(23)
    saved = oracle.ntt_max_L()
    try:
        for cap_lg in (10, 16, 22, 25):
            oracle.set_ntt_max_L(1 << cap_lg)
            ff.lib().ffg_set_ntt_max_L(1 << cap_lg)
            for _ in range(375):
                ba = int(2 ** rng.uniform(6, 28))
                sq = rng.random() < 0.3
                bb = ba if sq else int(2 ** min(28.0, max(6.0, math.log2(ba) + rng.uniform(-4, 4))))
                p = ff.plan(ba, bb, sq)
                o = oracle.plan(ba, bb, sq)
                assert (p["split"], p["width"], p["L"], p["lg"], p["r3"]) == (o.split, o.width, o.L, o.lg, o.r3), \
                    (cap_lg, ba, bb, sq, p)
                if o.split:
                    assert (p["ka"], p["kb"], p["Lbig"]) == (o.ka, o.kb, o.Lbig), (cap_lg, ba, bb, sq)
                else:
                    assert p["conv"] == o.conv
    finally:
        oracle.set_ntt_max_L(saved)
        ff.lib().ffg_set_ntt_max_L(saved)


def test_small_decimal_on_the_host(ff):
    """big_to_string below 16384 bits runs on the host (no GPU): every class of
    the reference's tests/dectest.py that fits -- zero, powers of ten and
    their neighbours, all-ones, chunk boundaries of 10^9 and 10^19, random
    numbers of every length up to the limit -- against Python's str."""
    import random

    from oracle import int_to_limbs
    rng = random.Random(7)
    xs = [0, 1, 9, 10, 999999999, 10**9, 10**9 + 1, 2**32 - 1, 2**32, 2**64 - 1, 2**64, 10**19 - 1, 10**19,
          10**19 + 1, 10**18 * 10**9, 2**16382 + 1, 2**16384 - 1 >> 1]
    for e in (1, 9, 18, 19, 38, 100, 1000, 2400, 4931):
        xs += [10**e - 1, 10**e, 10**e + 1]
    for bits in (1, 31, 32, 33, 63, 64, 65, 127, 128, 129, 1000, 4096, 8191, 8192, 12345, 16383):
        xs.append(rng.getrandbits(bits) | (1 << (bits - 1)))
        xs.append((1 << bits) - 1)
    for x in xs:
        assert x.bit_length() < 16384
        assert ff.big_to_string(int_to_limbs(x)) == str(x), x.bit_length()


def test_job_records_match_the_struct(ff):
    """device_jobs builds the same bytes as the ffg_job structs (include/ffg.h)."""
    jobs = [{"a": 1000 + i, "b": None if i % 3 == 0 else 2000 + i, "na": 100 + i, "nb": 200, "bits_a": 6400 + i,
             "bits_b": 12800, "out": 3000 + i, "square": i % 3 == 0, "method": ("plain", "ntt", "learned")[i % 3]}
            for i in range(50)]
    assert bytes(ff._device_jobs(jobs)) == ff.device_jobs(jobs).tobytes()
