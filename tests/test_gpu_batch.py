"""GPU parity of batched products (ffg_mul_batch_host / _device): many
independent products per call, grouped by plan into shared launches (the
reference multiplies them one at a time, e.g. one decimal level's products,
src/decimal.c:177-203).  Every method (the reference's thresholds, schoolbook,
big_mul_ntt's plan, lengths forced to 2^k and 3 * 2^k) gives the exact
product; the uneven stream of 4096 products (log-uniform 2^10..2^24 bits,
aspect up to 16:1) is checked exactly on a sample and by residues modulo
three 64-bit primes for every product."""
import numpy as np
import pytest

from fastfib_b200.workload import limbs_of_bits, uneven_products
from oracle import limbs_to_int

pytestmark = pytest.mark.gpu

PRIMES = (18446744073709551557, 18446744073709551533, 9223372036854775783)


@pytest.fixture(scope="module", autouse=True)
def _init(ff):
    ff.init(1 << 22)


def exact(pairs):
    return [limbs_to_int(a) * (limbs_to_int(a) if b is None else limbs_to_int(b)) for a, b in pairs]


@pytest.mark.parametrize("method", ["plain", "school", "ntt", "ntt_pow2", "ntt_r3"])
def test_methods_small(ff, method):
    pairs = uneven_products(seed=7, count=160, lo=6, hi=15)
    pairs += [(a, None) for a, _ in uneven_products(seed=8, count=40, lo=6, hi=15)]
    got = ff.mul_batch(pairs, method)
    for g, w, (a, b) in zip(got, exact(pairs), pairs):
        assert limbs_to_int(g) == w
        assert g.size == max(1, (w.bit_length() + 63) // 64)


def test_methods_mixed_and_edges(ff):
    rng = np.random.default_rng(3)
    pairs, methods = [], []
    names = ["plain", "school", "ntt", "ntt_pow2", "ntt_r3"]
    for i in range(250):
        ba, bb = int(2 ** rng.uniform(1, 17)), int(2 ** rng.uniform(1, 17))
        a = limbs_of_bits(rng, ba)
        b = None if i % 5 == 0 else limbs_of_bits(rng, bb)
        pairs.append((a, b))
        methods.append(names[i % 5])
    zero = np.zeros(3, dtype=np.uint64)
    ones = np.full(2000, 0xFFFFFFFFFFFFFFFF, dtype=np.uint64)
    padded = np.concatenate([ones[:300], np.zeros(9, dtype=np.uint64)])
    pairs += [(zero, ones), (ones, zero), (ones, None), (padded, ones), (np.array([1], dtype=np.uint64), ones)]
    methods += ["ntt", "school", "ntt_r3", "plain", "ntt_pow2"]
    got = ff.mul_batch(pairs, methods)
    for g, w in zip(got, exact(pairs)):
        assert limbs_to_int(g) == w


def test_uneven_stream_4096(ff):
    """The full uneven stream: residues modulo three primes for every product,
    exact comparison for a spread sample."""
    pairs = uneven_products(seed=4, count=4096)
    got = ff.mul_batch(pairs, "plain")
    for i, (g, (a, b)) in enumerate(zip(got, pairs)):
        x, y, z = limbs_to_int(a), limbs_to_int(b), limbs_to_int(g)
        for p in PRIMES:
            assert z % p == (x % p) * (y % p) % p, i
        assert z.bit_length() in (x.bit_length() + y.bit_length() - 1, x.bit_length() + y.bit_length()), i
    order = np.argsort([a.size + b.size for a, b in pairs])
    for i in list(order[::256]) + [int(order[-1])]:
        a, b = pairs[i]
        assert limbs_to_int(got[i]) == limbs_to_int(a) * limbs_to_int(b), i


def test_device_batch(ff):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    pairs = [(limbs_of_bits(rng, int(2 ** rng.uniform(8, 19))), limbs_of_bits(rng, int(2 ** rng.uniform(8, 19))))
             for _ in range(60)]
    dev = torch.device("cuda:0")
    keep, jobs = [], []
    for i, (a, b) in enumerate(pairs):
        ta = torch.from_numpy(a.view(np.int64)).to(dev)
        tb = torch.from_numpy(b.view(np.int64)).to(dev)
        sq = i % 4 == 0
        out = torch.full((a.size + (a.size if sq else b.size) + 1,), -1, dtype=torch.int64, device=dev)
        keep += [ta, tb, out]
        jobs.append({"a": ta.data_ptr(), "b": None if sq else tb.data_ptr(), "na": a.size,
                     "nb": a.size if sq else b.size, "bits_a": 64 * a.size, "bits_b": 64 * (a.size if sq else b.size),
                     "out": out.data_ptr(), "square": sq, "method": ("plain", "ntt", "school")[i % 3]})
    # on a stream of our own, after the uploads (NULL would be the library's stream)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    ff.mul_batch_device(jobs, side.cuda_stream)
    torch.cuda.synchronize()
    for i, ((a, b), j) in enumerate(zip(pairs, jobs)):
        out = keep[3 * i + 2].cpu().numpy().view(np.uint64)
        x = limbs_to_int(a)
        assert limbs_to_int(out) == x * (x if j["square"] else limbs_to_int(b))


@pytest.mark.parametrize("L", [6144, 8192, 12288, 16384])
@pytest.mark.parametrize("square", [True, False])
def test_large_group_one_cta(ff, L, square):
    """Groups of at least 64 products sharing a four-step plan of length up to
    16384 run one CTA per (product, prime) with the whole transform in
    shared memory: 64 products of each length (both length families,
    squares and distinct), against Python integers."""
    rng = np.random.default_rng(L + square)
    coeffs = int(0.85 * L)
    pairs = []
    for _ in range(64):
        if square:
            a = rng.integers(0, 2**64, size=(coeffs * 32 // 2 + 63) // 64, dtype=np.uint64)
            a[-1] |= np.uint64(1 << 63)
            pairs.append((a, None))
        else:
            a = rng.integers(0, 2**64, size=(coeffs * 32 // 3 + 63) // 64, dtype=np.uint64)
            b = rng.integers(0, 2**64, size=(2 * coeffs * 32 // 3 + 63) // 64, dtype=np.uint64)
            a[-1] |= np.uint64(1 << 63)
            b[-1] |= np.uint64(1 << 63)
            pairs.append((a, b))
    plan = ff.plan(64 * pairs[0][0].size, 64 * (pairs[0][0] if square else pairs[0][1]).size, square)
    assert plan["L"] == L and plan["kernel"] == 1, plan
    got = ff.mul_batch(pairs)
    assert [limbs_to_int(g) for g in got] == exact(pairs)


@pytest.mark.parametrize("n", [1 << 20, 1 << 22])
def test_microbench_sizes_every_length_family(ff, n):
    """The multiply microbench's large cases: distinct products and squares of
    random 2^20- and 2^22-limb operands at the reference's plan and with the
    transform length forced to 2^k and to 3 2^k (L up to 3 2^23).  The three
    results must agree limb for limb, and match the exact product modulo three
    64-bit primes and modulo 2^128 (the low limbs), with the exact bit length."""
    torch = pytest.importorskip("torch")
    ff.init(1 << 24)  # transform tables up to 2^25: no product here takes the split
    assert ff.plan(64 * n, 64 * n, False)["split"] == 0
    rng = np.random.default_rng(n + 11)
    a = rng.integers(0, 2**64, n, dtype=np.uint64)
    b = rng.integers(0, 2**64, n, dtype=np.uint64)
    a[-1] |= np.uint64(1 << 63)
    b[-1] |= np.uint64(1 << 62)
    xa, xb = limbs_to_int(a), limbs_to_int(b)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    for sq in (False, True):
        y = xa if sq else xb
        outs = []
        for m in ("ntt", "ntt_pow2", "ntt_r3"):
            out = torch.full((2 * n + 1,), -1, dtype=torch.int64, device="cuda")
            ff.mul_batch_device([{"a": da.data_ptr(), "b": (da if sq else db).data_ptr(), "na": n, "nb": n,
                                  "bits_a": 64 * n, "bits_b": 64 * n, "out": out.data_ptr(), "square": sq,
                                  "method": m}])
            torch.cuda.synchronize()
            outs.append(out.cpu().numpy().view(np.uint64).copy())
        assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
        z = limbs_to_int(outs[0])
        for p in PRIMES:
            assert z % p == (xa % p) * (y % p) % p
        assert z % 2**128 == (xa % 2**128) * (y % 2**128) % 2**128
        # bit length: the top two limbs of the operands fix it to within one
        # bit; the exact value follows from the product of the top parts
        top = (limbs_to_int(a[-2:]) * limbs_to_int((a if sq else b)[-2:])).bit_length()
        lo_bits = 64 * (n - 2) * 2
        assert z.bit_length() in (top + lo_bits, top + lo_bits + 1)
    del da, db
