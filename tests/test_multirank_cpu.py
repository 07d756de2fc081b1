"""CPU tests of the multi-rank logic (gloo, world size 2): frame sharding is
disjoint and the Monte Carlo counters are summed once at the end of a point."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    from gf2_b200.montecarlo import reduce_counters, shard_frame0
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        batch = 16
        mine = set()
        for b in range(5):
            f0 = shard_frame0(b, batch, rank, world)
            mine.update(range(f0, f0 + batch))
        c = torch.tensor([rank + 1, 10 * (rank + 1), 100], dtype=torch.int64)
        reduce_counters(c)
        q.put((rank, sorted(mine), c.tolist()))
    finally:
        dist.destroy_process_group()


def test_sharding_and_counter_reduction():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    a, b = set(res[0][1]), set(res[1][1])
    assert not (a & b) and len(a | b) == 2 * 5 * 16
    assert sorted(a | b) == list(range(160))
    for _, _, c in res:
        assert c == [3, 30, 200]


def test_wilson_interval():
    from gf2_b200.montecarlo import wilson
    lo, hi = wilson(0, 100)
    assert lo == 0.0 and 0.03 < hi < 0.04
    lo, hi = wilson(50, 100)
    assert 0.40 < lo < 0.41 and 0.59 < hi < 0.60
