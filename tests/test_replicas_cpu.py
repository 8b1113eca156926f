"""CPU: the multi-replica timing logic of bench.py on two gloo ranks
(the path does not shard; N GPUs run N independent replicas, the job's step
time is the slowest replica's)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(1.5 + rank, dist)          # rank 1 is slower
        dist.barrier()
        q.put((rank, t, bench.whole_job_value(100.0, t, world)))
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_weak_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]
    assert out[0][2] == pytest.approx(2 * 100.0 / 2.5)


def test_single_process_passthrough():
    assert bench.max_over_ranks(3.0, None) == 3.0
    assert bench.whole_job_value(10.0, 2.0, 1) == 5.0
