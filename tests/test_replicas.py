"""The multi-process replica path of bench.py (one process per GPU), run as two gloo
ranks on the CPU: disjoint scene batches per rank, barrier, and the whole-job
throughput (paths of all ranks over the slowest rank's time)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fumeng_b200.replicas import RankGroup, batch_indices


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        g = RankGroup(dist, "cpu")
        g.barrier()
        idx = batch_indices(rank, 3, 64)
        # rank r "renders" (r + 1) * 100 paths in (r + 1) * 10 ms
        value = g.throughput(paths=(rank + 1) * 100.0, elapsed_ms=(rank + 1) * 10.0)
        out.put((rank, idx, g.max(rank + 0.5), g.sum(rank + 1.0), value))
        g.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, i0, m0, s0, v0), (r1, i1, m1, s1, v1) = res
    assert (r0, r1) == (0, 1)
    assert i0 == [0, 1, 2] and i1 == [64, 65, 66] and not set(i0) & set(i1)
    assert m0 == m1 == 1.5 and s0 == s1 == 3.0
    # (100 + 200) paths over max(10, 20) ms = 15000 paths/s = 0.015 Mpaths/s on both ranks
    assert v0 == pytest.approx(0.015) and v1 == pytest.approx(0.015)


def test_single_process_group():
    g = RankGroup(None, "cpu")
    g.barrier()
    assert g.max(2.0) == 2.0 and g.sum(3.0) == 3.0
    assert g.throughput(1e6, 1000.0) == pytest.approx(1.0)
    assert batch_indices(0, 4) == [0, 1, 2, 3]
    assert torch.distributed.is_available()
