"""Sharding independent products over GPUs: one process per GPU, products
split by predicted cost, results gathered to one rank.

The reference multiplies independent products one at a time on one machine
(the halves of a decimal level, src/decimal.c:177-203; a user's stream of
big_mul calls).  Such products need no exchange while they are computed, so
they shard by product: every rank takes a share of the batch, runs it
through the batched device entry (ffg_mul_batch_device) on its own GPU, and
the products are gathered afterwards -- the only collective is that gather.

``partition`` balances the shares with the longest-processing-time rule over
a cost estimate per product: for an NTT product the transform length L of the
library's own plan (ffg_plan_select) times log2 L, for a product small enough
for schoolbook na * nb limb products scaled to the same units.

One product too large for one GPU's time budget shards by prime instead
(``mul_prime_sharded``): the three primes' transforms, pointwise products and
inverses are independent (src/mul_ntt.c:29-48 runs them one after another),
so each rank runs its primes' share (ffg_mul_residues), one broadcast per
prime from its owner completes every rank's residues -- 4 L bytes a prime,
the only exchange -- and the CRT (ffg_crt_residues) recombines them.
"""
from __future__ import annotations

import heapq
import math

import numpy as np

SCHOOL_MIN = 200  # below this short side the reference's thresholds take schoolbook / Karatsuba
SCHOOL_SCALE = 1.0 / 64  # limb products per transform-length unit (rough; only balance depends on it)


def product_cost(na: int, nb: int, square: bool = False, plan=None) -> float:
    """Predicted cost of one product of na x nb limbs, in arbitrary units
    (comparable between products).  plan: a callable (bits_a, bits_b, square)
    -> plan dict; by default the library's ffg_plan_select."""
    if min(na, nb) < SCHOOL_MIN:
        return max(1.0, na * nb * SCHOOL_SCALE)
    if plan is None:
        import fastfib_b200 as ff
        plan = ff.plan
    p = plan(64 * na, 64 * nb, square)
    L = p["Lbig"] if p["split"] else p["L"]
    return float(L) * math.log2(max(L, 2)) * (1.0 if square else 1.5)


def partition(costs, ranks: int) -> list[list[int]]:
    """Indices of each rank's share: products by decreasing cost, each to the
    rank with the least total so far (LPT); within a share, original order."""
    heap = [(0.0, r) for r in range(ranks)]
    shares = [[] for _ in range(ranks)]
    for i in sorted(range(len(costs)), key=lambda i: -costs[i]):
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shares]


def imbalance(costs, shares) -> float:
    """max over ranks of its total cost / the mean total, minus 1."""
    tot = [sum(costs[i] for i in s) for s in shares]
    mean = sum(tot) / len(tot)
    return max(tot) / mean - 1.0 if mean else 0.0


def gather_products(local: dict[int, np.ndarray], count: int, group=None, dst: int = 0, device=None):
    """Collects every rank's products (index -> limbs) on rank dst, which gets
    the list of all `count` products in index order; other ranks get None.
    Uses torch.distributed: the products are limb arrays of different
    lengths, sent as one flat buffer per rank, staged on `device` (a CUDA
    device for NCCL; by default the backend decides)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
            else torch.device("cpu")
    idx = np.array(sorted(local), dtype=np.int64)
    lens = np.array([local[i].size for i in idx], dtype=np.int64)
    flat = np.concatenate([local[i] for i in idx]).view(np.int64) if idx.size else np.zeros(0, np.int64)
    # sizes first (every rank learns every rank's count and length), then data
    head = torch.tensor([idx.size, flat.size], dtype=torch.int64, device=device)
    heads = [torch.zeros(2, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(heads, head, group=group)
    heads = [h.cpu() for h in heads]
    n_max = max(int(h[0]) for h in heads)
    f_max = max(int(h[1]) for h in heads)
    meta = torch.full((2, max(1, n_max)), -1, dtype=torch.int64)
    meta[0, :idx.size] = torch.from_numpy(idx)
    meta[1, :idx.size] = torch.from_numpy(lens)
    data = torch.zeros(max(1, f_max), dtype=torch.int64)
    data[:flat.size] = torch.from_numpy(flat.copy())
    meta, data = meta.to(device), data.to(device)
    metas = [torch.zeros_like(meta) for _ in range(world)] if rank == dst else None
    datas = [torch.zeros_like(data) for _ in range(world)] if rank == dst else None
    dist.gather(meta, metas, dst=dst, group=group)
    dist.gather(data, datas, dst=dst, group=group)
    if rank != dst:
        return None
    out = [None] * count
    for r in range(world):
        n = int(heads[r][0])
        m, d = metas[r].cpu().numpy(), datas[r].cpu().numpy().view(np.uint64)
        o = 0
        for k in range(n):
            i, ln = int(m[0, k]), int(m[1, k])
            out[i] = d[o: o + ln].copy()
            o += ln
    return out


def mul_batch_sharded(pairs, method: str = "plain", group=None, dst: int = 0, mul=None):
    """The products of pairs ((a, b), b None squares) split over the ranks of
    group by predicted cost, each rank computing its share with `mul` (by
    default the library's batched entry, fastfib_b200.mul_batch, on this
    rank's GPU), gathered on rank dst (the list of products in order; None
    elsewhere).  Returns (products or None, this rank's indices)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    costs = [product_cost(a.size, (a if b is None else b).size, b is None) for a, b in pairs]
    share = partition(costs, world)[rank]
    if mul is None:
        import fastfib_b200 as ff

        def mul(ps):
            return ff.mul_batch(ps, method)
    got = mul([pairs[i] for i in share]) if share else []
    local = {i: np.asarray(g, dtype=np.uint64) for i, g in zip(share, got)}
    return gather_products(local, len(pairs), group=group, dst=dst), share


def prime_shares(world: int) -> list[tuple[int, int]]:
    """(prime0, nprimes) of every rank when one product's three primes are
    spread over `world` ranks: contiguous ranges as even as three allows
    (two ranks: one prime and two); ranks past the third get (0, 0)."""
    used = min(world, 3)
    out = []
    for r in range(world):
        if r >= used:
            out.append((0, 0))
        else:
            lo, hi = 3 * r // used, 3 * (r + 1) // used
            out.append((lo, hi - lo))
    return out


def _bits(x: np.ndarray) -> int:
    nz = np.flatnonzero(x)
    if nz.size == 0:
        return 0
    top = int(nz[-1])
    return 64 * top + int(x[top]).bit_length()


def mul_prime_sharded(a, b=None, group=None, dst=None, residues=None, crt=None, plan=None):
    """The product a * b (b None: a squared) with its three primes spread over
    the ranks of group (prime_shares).  Each rank computes its primes'
    residues, one broadcast per prime from the rank that owns it fills in the
    others, and the CRT recombines all three on rank dst (every rank when dst
    is None); other ranks return None.  The product is returned as limbs.

    By default the work runs on this rank's GPU through the library
    (ffg_mul_residues / ffg_crt_residues) and the residues stay in device
    memory for the broadcasts (NCCL).  The tests pass the oracle's instead:
    residues(a, b, square, k) -> prime k's L words, crt(y (3 x L), a, b,
    square) -> limbs, and plan(bits_a, bits_b, square) -> {"L", "width",
    "kernel", "split"}; the buffers then live on the CPU (gloo)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    square = b is None
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = a if square else np.ascontiguousarray(b, dtype=np.uint64)
    bits_a, bits_b = _bits(a), _bits(b)
    if bits_a == 0 or bits_b == 0:
        raise ValueError("mul_prime_sharded: a zero factor")
    library = residues is None
    if plan is None:
        import fastfib_b200 as ff
        plan = ff.plan
    pl = plan(bits_a, bits_b, square)
    if pl["split"] or not pl["kernel"]:
        raise ValueError("mul_prime_sharded: four-step plans only (not a one-CTA length or a split product)")
    L = int(pl["L"])
    prime0, nprimes = prime_shares(world)[rank]
    shares = prime_shares(world)
    if not library:
        y = torch.zeros((3, L), dtype=torch.int32)
        for k in range(prime0, prime0 + nprimes):
            y[k] = torch.from_numpy(np.asarray(residues(a, b, square, k), dtype=np.uint32).view(np.int32))
        _broadcast_primes(y, shares, group)
        if dst is not None and rank != dst:
            return None
        return np.asarray(crt(y.numpy().view(np.uint32), a, b, square), dtype=np.uint64)
    import fastfib_b200 as ff
    dev = torch.device("cuda", torch.cuda.current_device())
    # a stream of our own: the library runs on the stream it is given (NULL,
    # the legacy default stream's handle, would mean its own stream), and the
    # uploads, the broadcasts (NCCL waits on the current stream) and the CRT
    # must all be ordered on it
    side = torch.cuda.Stream(device=dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        stream = side.cuda_stream
        da = torch.from_numpy(a.view(np.int64)).to(dev)
        db = da if square else torch.from_numpy(b.view(np.int64)).to(dev)
        y = torch.zeros((3, L), dtype=torch.int32, device=dev)
        if nprimes:
            ff.mul_residues(y.data_ptr(), da.data_ptr(), a.size, bits_a, db.data_ptr(), b.size, bits_b, square,
                            prime0, nprimes, stream)
        _broadcast_primes(y, shares, group)
        if dst is not None and rank != dst:
            side.synchronize()
            return None
        out = torch.empty(a.size + b.size + 1, dtype=torch.int64, device=dev)
        ff.crt_residues(out.data_ptr(), y.data_ptr(), a.size, bits_a, b.size, bits_b, square, stream)
        res = out.cpu().numpy().view(np.uint64)
    return res


def _broadcast_primes(y, shares, group):
    """Every prime's row of y from the rank that owns it; every rank takes the
    same three broadcasts, in order."""
    import torch.distributed as dist
    for k in range(3):
        owner = next(r for r, (p0, n) in enumerate(shares) if p0 <= k < p0 + n)
        src = dist.get_global_rank(group, owner) if group is not None else owner
        dist.broadcast(y[k], src=src, group=group)
