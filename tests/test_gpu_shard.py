"""GPU tests of one product sharded by prime (ffg_mul_residues /
ffg_crt_residues, fastfib_b200.shard.mul_prime_sharded): every prime's
residues computed alone match the oracle's convolution modulo that prime
word for word, the CRT of the three slices is exactly the product
ffg_mul_device writes and the Python product, for each way of splitting the
primes, for squares, distinct products, both length families and the row
kernels' shapes; the entry points refuse the plans they do not take."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _cap(ff):
    ff.init(1 << 22)  # transforms up to 2^23 words: none of these products splits
    # every test on a stream of its own: the library runs on the stream it is
    # given (NULL, the legacy default stream's handle, means its own stream),
    # so uploads, library calls and comparisons are ordered on this one
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        yield
    side.synchronize()


def _bits(x):
    from fastfib_b200.shard import _bits
    return _bits(x)


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint64).view(np.int64)).cuda()


def _stream():
    """The test's stream (never the legacy default stream)."""
    s = torch.cuda.current_stream().cuda_stream
    assert s, "run under the test's own stream"
    return s


def _residues(ff, a, b, square, splits):
    """y (3, L) filled by one ffg_mul_residues call per (prime0, nprimes)."""
    b = a if square else b
    pl = ff.plan(_bits(a), _bits(b), square)
    da, db = _dev(a), _dev(b)
    y = torch.zeros((3, pl["L"]), dtype=torch.int32, device="cuda")
    for p0, n in splits:
        ff.mul_residues(y.data_ptr(), da.data_ptr(), a.size, _bits(a), db.data_ptr(), b.size, _bits(b), square,
                        p0, n, _stream())
    return pl, y


CASES = [  # (limbs of a, limbs of b or None for a square)
    (3000, 2100),     # L = 3 2^12 (radix 3)
    (2600, None),     # a square
    (20000, 17000),   # L = 2^16
    (70000, None),    # L = 3 2^16, a square
    (300000, 250000), # L = 2^20
]


@pytest.mark.parametrize("na,nb", CASES)
def test_each_prime_alone_and_the_crt(ff, oracle, na, nb):
    rng = np.random.default_rng(na)
    a = rng.integers(0, 2**63, na, dtype=np.uint64) | np.uint64(1)
    b = None if nb is None else rng.integers(0, 2**63, nb, dtype=np.uint64)
    square = b is None
    bb = a if square else b
    pl, y = _residues(ff, a, b, square, [(0, 1), (1, 1), (2, 1)])
    assert pl["kernel"] == 1 and not pl["split"]
    w, L = pl["width"], pl["L"]
    conv = (_bits(a) + w - 1) // w + (_bits(bb) + w - 1) // w - 1
    yh = y.cpu().numpy().view(np.uint32)
    if na <= 70000:  # the oracle's textbook transform takes seconds beyond
        oracle.ntt_init(1 << 20)
        for k in range(3):
            want = oracle.residues(a, bb, w, L, k, square)
            assert np.array_equal(yh[k, :conv], want[:conv]), k
    out = torch.empty(a.size + bb.size + 1, dtype=torch.int64, device="cuda")
    ff.crt_residues(out.data_ptr(), y.data_ptr(), a.size, _bits(a), bb.size, _bits(bb), square, _stream())
    ref = torch.empty_like(out)
    da, db = _dev(a), _dev(bb)  # held: a temporary's memory would be reused by the next upload
    ff.mul_device(ref.data_ptr(), da.data_ptr(), a.size, _bits(a), db.data_ptr(), bb.size, _bits(bb), square,
                  _stream())
    assert torch.equal(out, ref)
    if na <= 70000:
        from oracle import limbs_to_int
        got = limbs_to_int(out.cpu().numpy().view(np.uint64))
        assert got == limbs_to_int(a) * limbs_to_int(bb)


@pytest.mark.parametrize("splits", [[(0, 3)], [(0, 2), (2, 1)], [(0, 1), (1, 2)], [(2, 1), (0, 1), (1, 1)]])
def test_every_split_of_the_primes(ff, splits):
    rng = np.random.default_rng(5)
    a = rng.integers(0, 2**64, 40000, dtype=np.uint64)
    b = rng.integers(0, 2**64, 33000, dtype=np.uint64)
    _, y = _residues(ff, a, b, False, splits)
    _, y3 = _residues(ff, a, b, False, [(0, 3)])
    assert torch.equal(y, y3)


def test_refusals(ff):
    rng = np.random.default_rng(6)
    small = rng.integers(0, 2**63, 100, dtype=np.uint64)  # a one-CTA length
    da = _dev(small)
    y = torch.zeros((3, 1 << 14), dtype=torch.int32, device="cuda")
    with pytest.raises(ff.FfgError):
        ff.mul_residues(y.data_ptr(), da.data_ptr(), small.size, _bits(small), da.data_ptr(), small.size,
                        _bits(small), True, 0, 3, _stream())
    a = rng.integers(0, 2**63, 3000, dtype=np.uint64)
    db = _dev(a)
    for p0, n in [(0, 0), (1, 3), (3, 1), (2, 2)]:
        with pytest.raises(ff.FfgError):
            ff.mul_residues(y.data_ptr(), db.data_ptr(), a.size, _bits(a), db.data_ptr(), a.size, _bits(a),
                            True, p0, n, _stream())
    cap = ff.lib().ffg_ntt_max_L()
    try:  # a split product (past the transform cap)
        ff.lib().ffg_set_ntt_max_L(1 << 12)
        with pytest.raises(ff.FfgError):
            ff.mul_residues(y.data_ptr(), db.data_ptr(), a.size, _bits(a), db.data_ptr(), a.size, _bits(a),
                            True, 0, 3, _stream())
    finally:
        ff.lib().ffg_set_ntt_max_L(cap)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_mul_prime_sharded_through_nccl(ff):
    """The library path of mul_prime_sharded end to end: its residues on the
    device, the broadcasts over NCCL (one rank: this run has one GPU), the CRT
    on the device."""
    import torch.distributed as dist
    from fastfib_b200.shard import mul_prime_sharded
    from oracle import limbs_to_int
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        rng = np.random.default_rng(8)
        a = rng.integers(0, 2**64, 9000, dtype=np.uint64)
        b = rng.integers(0, 2**64, 7000, dtype=np.uint64)
        got = mul_prime_sharded(a, b)
        assert limbs_to_int(got) == limbs_to_int(a) * limbs_to_int(b)
        got = mul_prime_sharded(a)
        assert limbs_to_int(got) == limbs_to_int(a) ** 2
    finally:
        dist.destroy_process_group()
