"""CPU test of the multi-GPU path of bench.py (replicas: one process per GPU,
no data exchange beyond the timing): two gloo ranks on 127.0.0.1 reduce
their totals with the same job_ms the bench uses over NCCL, and every rank
gets the max over ranks divided by steps * world."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    totals = [10.0 + 5 * rank, 20.0 - 3 * rank]  # rank 1 slower on device, rank 0 on the host
    got = bench.job_ms(totals, steps=4, world=world, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def test_job_ms_max_over_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    for r in range(2):
        assert res[r] == [15.0 / 8, 20.0 / 8]


def test_job_ms_one_rank():
    import bench
    assert bench.job_ms([8.0, 12.0], steps=4, world=1) == [2.0, 3.0]
