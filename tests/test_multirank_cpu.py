"""CPU tests of the multi-rank logic (gloo, world size 2): frame sharding is
disjoint, the Monte Carlo counters are summed once at the end of a point, and
data-parallel training of the learned decoder (one gradient all-reduce per
step) applies the same updates as training on one rank."""
import os
import socket

import numpy as np
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


def _adam(p, g, m, v, step, lr=1e-2, b1=0.9, b2=0.999, eps=1e-8):
    m[:] = b1 * m + (1 - b1) * g
    v[:] = b2 * v + (1 - b2) * g * g
    p[:] = np.clip(p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps), -4, 4)


def _train_cpu(rank, world, steps, batch, T, layered, reduce=None):
    """Data-parallel training steps of NmsTrainer's host logic (batch_plan, the
    shard rescale and the gradient all-reduce of gf2_b200.learned) with the FP64
    oracle as the gradient kernel and a NumPy Adam step."""
    import torch

    from gf2_b200.learned import batch_plan, data_parallel_reduce
    from oracle import pyoracle
    oc = pyoracle.Code.dvbt2(1, 5)
    L = oc.layers
    P = np.concatenate([np.full(T * L, 0.9), np.full(T * L, 0.1)])
    M, V = np.zeros_like(P), np.zeros_like(P)
    losses = []
    for s in range(steps):
        f0, cnt, eb = batch_plan(3, s * batch, batch, (2.5, 3.5), rank, world)
        _, cw, llr = oc.channel(3, f0, cnt, eb)
        loss, ga, gb, _ = oc.nms_loss_grad(llr, cw, T, P[:T * L], P[T * L:], layered=layered)
        flat = torch.from_numpy(np.concatenate([ga, gb, [loss]]))
        data_parallel_reduce(flat, cnt, batch) if reduce is None else reduce(flat, cnt, batch)
        g = flat.numpy()
        losses.append(float(g[-1]))
        _adam(P, g[:-1], M, V, s + 1)
    return P, losses


def _dp_worker(rank, world, port, q, layered):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P, losses = _train_cpu(rank, world, 3, 4, 3, layered)
        q.put((rank, P.tolist(), losses))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("layered", [False, True])
def test_data_parallel_training_equals_one_rank(layered):
    """Two gloo ranks on half batches apply the same Adam updates as one rank on
    the full batch (FP64 oracle gradients; the all-reduce sums the shards'
    rescaled gradient sums, so the results agree to rounding)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, q, layered)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    P1, l1 = _train_cpu(0, 1, 3, 4, 3, layered)
    for _, P, losses in res:
        assert np.allclose(P, P1, rtol=1e-10, atol=1e-12)
        assert np.allclose(losses, l1, rtol=1e-10)
    assert np.abs(P1 - np.concatenate([np.full(len(P1) // 2, 0.9), np.full(len(P1) // 2, 0.1)])).max() > 1e-3
