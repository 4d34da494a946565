"""CPU tests of the sharding over GPUs (fastfib_b200/shard.py): the cost
partition of the uneven product stream over 2..8 ranks; the sharded batch
with its gather on two gloo ranks, each rank's share computed by the oracle,
whose union on rank 0 must be exactly the single-rank result; and one product
sharded by prime over two and three gloo ranks, each rank computing only its
primes' residues (the oracle's), the product recombined on every rank."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _costs(ff, pairs):
    from fastfib_b200.shard import product_cost
    ff.lib().ffg_set_ntt_max_L(1 << 25)
    return [product_cost(a.size, (a if b is None else b).size, b is None) for a, b in pairs]


def test_partition_of_the_uneven_stream(ff):
    from fastfib_b200.shard import imbalance, partition
    from fastfib_b200.workload import uneven_sizes
    sizes = uneven_sizes(seed=4, count=4096)
    pairs = [(np.zeros((x + 63) // 64, np.uint64), np.zeros((y + 63) // 64, np.uint64)) for x, y in sizes]
    costs = _costs(ff, pairs)
    for ranks in (2, 3, 4, 8):
        shares = partition(costs, ranks)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(pairs)))  # every product once
        assert imbalance(costs, shares) < 0.10, ranks


def test_partition_edge_cases():
    from fastfib_b200.shard import imbalance, partition
    assert partition([], 3) == [[], [], []]
    assert partition([5.0], 2) in ([[0], []], [[], [0]])
    shares = partition([1.0] * 10, 4)
    assert sorted(len(s) for s in shares) == [2, 2, 3, 3]
    assert imbalance([1.0] * 8, partition([1.0] * 8, 4)) == 0.0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pairs():
    from fastfib_b200.workload import uneven_products
    pairs = uneven_products(seed=9, count=120, lo=6, hi=15)
    return pairs + [(a, None) for a, _ in uneven_products(seed=10, count=30, lo=6, hi=14)]


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import fastfib_b200 as ff
        from fastfib_b200.shard import mul_batch_sharded, partition, product_cost
        from oracle import Oracle
        ff.lib().ffg_set_ntt_max_L(1 << 25)
        o = Oracle()
        o.ntt_init(1 << 16)
        pairs = _pairs()

        def mul(ps):  # this rank's share, on the CPU checker
            return [o.mul(a, b) if b is not None else o.mul(a) for a, b in ps]

        got, share = mul_batch_sharded(pairs, group=None, dst=0, mul=mul)
        costs = [product_cost(a.size, (a if b is None else b).size, b is None) for a, b in pairs]
        assert share == partition(costs, world)[rank]
        res = None
        if rank == 0:
            want = mul(pairs)
            res = all(np.array_equal(g, w) for g, w in zip(got, want)) and len(got) == len(want)
        else:
            res = got is None
        dist.barrier()
        q.put((rank, res, len(share)))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_on_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = {}
    for _ in range(2):
        r, ok, n = q.get(timeout=10)
        res[r] = (ok, n)
    assert res[0][0] is True and res[1][0] is True
    assert res[0][1] + res[1][1] == len(_pairs()) and res[0][1] > 0 and res[1][1] > 0


def test_prime_shares():
    from fastfib_b200.shard import prime_shares
    assert prime_shares(1) == [(0, 3)]
    assert prime_shares(2) == [(0, 1), (1, 2)]
    assert prime_shares(3) == [(0, 1), (1, 1), (2, 1)]
    assert prime_shares(5)[3:] == [(0, 0), (0, 0)]
    for w in range(1, 9):  # every prime owned by exactly one rank
        owned = [k for p0, n in prime_shares(w) for k in range(p0, p0 + n)]
        assert sorted(owned) == [0, 1, 2]


def _prime_rank(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from fastfib_b200.shard import _bits, mul_prime_sharded, prime_shares
        from oracle import Oracle, int_to_limbs, limbs_to_int
        o = Oracle()
        o.ntt_init(1 << 16)
        rng = np.random.default_rng(21)
        cases = [(rng.integers(0, 2**63, 3000, dtype=np.uint64), rng.integers(0, 2**63, 2100, dtype=np.uint64)),
                 (rng.integers(0, 2**63, 2600, dtype=np.uint64), None),
                 (int_to_limbs((1 << (64 * 1500)) - 1), int_to_limbs((1 << (64 * 1700)) - 1))]
        calls = []

        def plan(bits_a, bits_b, square):
            p = o.plan(bits_a, bits_b, square)
            return {"L": p.L, "width": p.width, "split": p.split, "kernel": 1}

        def residues(a, b, square, k):
            calls.append(k)
            p = o.plan(_bits(a), _bits(b), square)
            return o.residues(a, b, p.width, p.L, k, square)

        def crt(y, a, b, square):
            p = o.plan(_bits(a), _bits(b), square)
            ca = (_bits(a) + p.width - 1) // p.width
            cb = (_bits(b) + p.width - 1) // p.width
            return o.crt_residues(y, p.L, ca + cb - 1, p.width, a.size + b.size + 1)

        ok = True
        for a, b in cases:
            got = mul_prime_sharded(a, b, residues=residues, crt=crt, plan=plan)
            want = limbs_to_int(a) * limbs_to_int(a if b is None else b)
            ok = ok and limbs_to_int(got) == want
        p0, n = prime_shares(world)[rank]
        mine = sorted(set(calls)) == list(range(p0, p0 + n)) and len(calls) == n * len(cases)
        dist.barrier()
        q.put((rank, ok, mine))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_prime_sharded_product_on_gloo_ranks(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_prime_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = {}
    for _ in range(world):
        r, ok, mine = q.get(timeout=10)
        res[r] = (ok, mine)
    assert all(ok and mine for ok, mine in res.values()), res


def test_prime_sharded_one_rank_and_refusals(oracle):
    """One gloo rank computes all three primes itself; plans prime sharding
    does not take (a one-CTA length, a split product) and zero factors are
    refused before any collective."""
    import torch.distributed as dist
    from fastfib_b200.shard import _bits, mul_prime_sharded
    from oracle import limbs_to_int
    oracle.ntt_init(1 << 16)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        def plan(bits_a, bits_b, square, kernel=1, split=None):
            p = oracle.plan(bits_a, bits_b, square)
            return {"L": p.L, "width": p.width, "split": p.split if split is None else split, "kernel": kernel}

        def residues(a, b, square, k):
            p = oracle.plan(_bits(a), _bits(b), square)
            return oracle.residues(a, b, p.width, p.L, k, square)

        def crt(y, a, b, square):
            p = oracle.plan(_bits(a), _bits(b), square)
            conv = (_bits(a) + p.width - 1) // p.width + (_bits(b) + p.width - 1) // p.width - 1
            return oracle.crt_residues(y, p.L, conv, p.width, a.size + b.size + 1)

        rng = np.random.default_rng(3)
        a = rng.integers(0, 2**64, 1500, dtype=np.uint64)
        b = rng.integers(0, 2**64, 1100, dtype=np.uint64)
        got = mul_prime_sharded(a, b, residues=residues, crt=crt, plan=plan)
        assert limbs_to_int(got) == limbs_to_int(a) * limbs_to_int(b)
        with pytest.raises(ValueError):  # a one-CTA length
            mul_prime_sharded(a, b, residues=residues, crt=crt, plan=lambda *x: plan(*x, kernel=0))
        with pytest.raises(ValueError):  # a split product
            mul_prime_sharded(a, b, residues=residues, crt=crt, plan=lambda *x: plan(*x, split=1))
        with pytest.raises(ValueError):  # a zero factor
            mul_prime_sharded(np.zeros(4, np.uint64), b, residues=residues, crt=crt, plan=plan)
    finally:
        dist.destroy_process_group()
