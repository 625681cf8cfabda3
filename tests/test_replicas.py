"""Replica aggregation over two gloo ranks on the CPU: the job rate is the
units of all ranks over the slowest rank's time, as bench.py reports it."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, seconds, units, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from mcdfci_b200.replicas import max_over_ranks, replica_rate

        q.put((rank, max_over_ranks(seconds[rank], dist), replica_rate(units, seconds[rank], world, dist)))
    finally:
        dist.destroy_process_group()


def test_replica_rate_two_gloo_ranks():
    world, units = 2, 3200.0
    seconds = [0.25, 0.40]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, seconds, units, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, mx, rate in got:
        assert mx == max(seconds)
        assert rate == pytest.approx(world * units / max(seconds), rel=0, abs=1e-9)


def test_replica_rate_single_process():
    from mcdfci_b200.replicas import replica_rate

    assert replica_rate(100.0, 0.5, 1) == 200.0
    with pytest.raises(ValueError):
        replica_rate(1.0, 0.0, 1)
