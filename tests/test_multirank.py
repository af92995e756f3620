"""Multi-rank plumbing of bench.py on CPU: two gloo ranks.

The GF solves shard across ranks with no collective in the data path; the
only collectives are the barrier and the max-over-ranks timing reduction.
These tests run those pieces as real torch.distributed processes on the
host (no GPU), including a rank that never joins.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, q):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        if mode == "absent" and rank == 1:
            q.put((rank, "absent", None))
            return  # this rank never joins the group
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=8))
        if mode == "shard":
            batch, steps = 3, 4
            mine = []
            for step in range(steps):
                f = bench.rank_first_source(step, world, rank, batch)
                mine += list(range(f, f + batch))
            got = bench.reduce_max(float(10 * rank + 1), dist, "cpu")
            dist.barrier()
            q.put((rank, mine, got))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent, which asserts on it
        q.put((rank, "error", type(e).__name__ + ": " + str(e)[:200]))


def _run(mode, world=2, timeout=60):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = {}
    for _ in range(world):
        r, a, b = q.get(timeout=timeout)
        out[r] = (a, b)
    for p in ps:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return out


def test_sources_are_disjoint_and_timing_is_max_over_ranks():
    out = _run("shard")
    s0, m0 = out[0]
    s1, m1 = out[1]
    assert not set(s0) & set(s1)
    assert sorted(s0 + s1) == list(range(2 * 3 * 4))  # every source exactly once
    assert m0 == m1 == 11.0  # max(1, 11)


def test_missing_rank_ends_in_an_error_not_a_hang():
    out = _run("absent", timeout=90)
    assert out[1][0] == "absent"
    assert out[0][0] == "error"
