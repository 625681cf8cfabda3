"""The curve spread over ranks (mcdfci_b200.curve) on two and three gloo ranks
on the CPU: every point is solved by exactly one rank (i mod world), and rank
0 receives all results in point order.  The solving step is a stand-in that
records which rank solved which point, so no GPU is needed; the GPU step
itself is the batch tested in test_gpu_batch.py."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mcdfci_b200.curve import gather_results, share, solve_curve


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, n, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        def solve_share(points):
            return {i: {"energy": -100.0 - 0.5 * i, "rank": rank} for i in points}

        out = solve_curve(n, solve_share, dist)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_curve_points_dealt_and_gathered(world):
    n = 32
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = got[0]
    assert len(out) == n
    for i, r in enumerate(out):
        assert r["energy"] == -100.0 - 0.5 * i
        assert r["rank"] == i % world
    for rank in range(1, world):
        assert got[rank] is None


def test_share_and_gather_single_process():
    assert share(5, 0, 2) == [0, 2, 4] and share(5, 1, 2) == [1, 3]
    with pytest.raises(ValueError):
        share(4, 2, 2)
    out = gather_results({1: {"e": 1}, 0: {"e": 0}}, 2)
    assert [r["e"] for r in out] == [0, 1]
    with pytest.raises(ValueError):
        gather_results({0: {"e": 0}}, 2)
