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
        if mode == "kh":
            # KH targets split across ranks: surface traces only on rank 0,
            # broadcast once; the blocks gathered on every rank
            import numpy as np

            from acoustic_disguising_b200.shard import kh_sharded
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import pyoracle

            c = _kh_case()
            def compute(sp, sn, q, f, rp, rn):  # the oracle stands in for the GPU kernel
                return pyoracle.kh_pressure(sp, sn, rp, q, f, c["dt"], c["sigma"], 343.0,
                                            c["aq"], c["af"], mode=1).astype(np.float32)
            mine = rank == 0
            out = kh_sharded(compute, c["sp"] if mine else None, c["sn"] if mine else None,
                             c["q"] if mine else None, c["f"] if mine else None, c["rp"],
                             dist=dist)
            q.put((rank, out, None))
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


def _kh_case(ns=40, nr=23, nt=300):
    import numpy as np

    rng = np.random.default_rng(5)
    i = np.arange(ns)
    z = 1 - (2 * i + 1) / ns
    th = np.pi * (3 - np.sqrt(5)) * i
    rxy = np.sqrt(1 - z * z)
    sn = np.stack([rxy * np.cos(th), rxy * np.sin(th), z], 1)
    rp = rng.standard_normal((nr, 3))
    rp *= 0.9 / np.linalg.norm(rp, axis=1, keepdims=True)
    q = np.asfortranarray(rng.standard_normal((nt, ns)).astype(np.float32))
    f = np.asfortranarray(rng.standard_normal((nt, ns)).astype(np.float32))
    return dict(sp=0.25 * sn, sn=sn, rp=rp, q=q, f=f, dt=5e-6,
                sigma=np.sqrt(np.log(2.0)) / (2 * np.pi * 20e3), aq=-1e-6, af=-2e-6)


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


def test_kh_targets_split_across_ranks_gather_to_the_full_sum():
    """Two gloo ranks: rank 0 alone holds the surface traces; each rank sums
    its block of targets; every rank ends with the full (nt, nr) result,
    equal to the sum over all targets in one process."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    out = _run("kh", timeout=120)
    c = _kh_case()
    full = pyoracle.kh_pressure(c["sp"], c["sn"], c["rp"], c["q"], c["f"], c["dt"], c["sigma"],
                                343.0, c["aq"], c["af"], mode=1).astype(np.float32)
    for r in (0, 1):
        got = out[r][0]
        assert isinstance(got, np.ndarray), out[r]
        assert got.shape == full.shape and np.array_equal(got, full)


@pytest.mark.parametrize("nr,world", [(16384, 8), (23, 2), (5, 4), (3, 8), (0, 3)])
def test_target_blocks_cover_every_target_once(nr, world):
    from acoustic_disguising_b200.shard import target_block

    blocks = [target_block(nr, r, world) for r in range(world)]
    assert blocks[0][0] == 0 and blocks[-1][1] == nr
    assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
    sizes = [e - b for b, e in blocks]
    assert max(sizes) - min(sizes) <= 1
