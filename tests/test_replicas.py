"""Several GPUs (replicas): the timing reduction and the ensemble member split,
on two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from spoc_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms, units = replicas.reduce_throughput(10.0 * (rank + 1), 100.0 + rank, world)
        share = replicas.member_share(11, rank, world)
        out.put((rank, ms, units, share))
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_and_split():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, units, _ in res:
        assert ms == 20.0          # the slowest rank's time
        assert units == 201.0      # both ranks' work
    shares = [r[3] for r in res]
    assert sorted(shares[0] + shares[1]) == list(range(11))
    assert not set(shares[0]) & set(shares[1])


def test_single_rank_is_local():
    assert replicas.reduce_throughput(3.0, 7.0, 1) == (3.0, 7.0)
    assert replicas.member_share(5, 0, 1) == [0, 1, 2, 3, 4]
