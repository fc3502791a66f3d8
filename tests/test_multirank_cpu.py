"""Multi-GPU host logic on the CPU (no GPU): the rod partition that shards a
batch across ranks, and the cross-rank reductions, run as two gloo ranks."""
import os
import socket

import numpy as np
import pytest


def test_partition_balanced_complete_deterministic():
    from elasticapp_b200 import dist
    rng = np.random.default_rng(5)
    w = rng.integers(32, 513, size=5000)
    for k in (1, 2, 4, 8):
        p = dist.partition(w, k)
        assert p.min() >= 0 and p.max() < k
        sums = np.bincount(p, weights=w, minlength=k)
        assert sums.sum() == w.sum()
        assert sums.max() - sums.min() <= w.max()  # within one item
        assert np.array_equal(p, dist.partition(w, k))
    # the largest differencing method beats naive round robin
    rr = np.arange(len(w)) % 8
    s_rr = np.bincount(rr, weights=w, minlength=8)
    s_kk = np.bincount(dist.partition(w, 8), weights=w, minlength=8)
    assert s_kk.max() - s_kk.min() <= s_rr.max() - s_rr.min()


def test_partition_known_answer():
    from elasticapp_b200 import dist
    # {8, 7, 6, 5, 4}: the largest differencing method's two-way split is
    # {8, 6} / {7, 5, 4} (sums 14 and 16)
    p = dist.partition([8, 7, 6, 5, 4], 2)
    sums = sorted(np.bincount(p, weights=[8, 7, 6, 5, 4], minlength=2))
    assert sums == [14.0, 16.0]
    with pytest.raises(Exception):
        dist.partition([1, -2], 2)


def test_shard_keeps_per_rod_data_aligned():
    from elasticapp_b200 import dist, workloads as W
    wl = W.mixed_batch(n_rods=64, seed=3)
    parts = dist.partition(wl.n_elements, 3)
    shards = [dist.shard(wl, r, 3, parts) for r in range(3)]
    assert sum(len(s.rods) for s in shards) == 64
    for r, s in enumerate(shards):
        idx = np.flatnonzero(parts == r)
        for j, i in enumerate(idx):
            assert s.rods[j] is wl.rods[i]
            assert s.velocities[j] is wl.velocities[i]
            assert s.rest_curvature[j] is wl.rest_curvature[i]
            assert np.array_equal(s.end_torque[j], wl.end_torque[i])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as tdist

    from elasticapp_b200 import dist, workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wl = W.uneven_batch(n_rods=200, seed=1002)
        mine = dist.shard(wl, rank, world)
        elems = dist.sum_over_ranks(mine.total_elements)
        worst = dist.max_over_ranks(float(rank + 1))
        tdist.barrier()
        q.put((rank, len(mine.rods), mine.total_elements, elems, worst))
    finally:
        tdist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    import torch.multiprocessing as mp
    from elasticapp_b200 import workloads as W
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    total = W.uneven_batch(n_rods=200, seed=1002).total_elements
    got.sort()
    assert sum(g[1] for g in got) == 200
    assert sum(g[2] for g in got) == total
    for g in got:
        assert g[3] == total and g[4] == 2.0
    assert abs(got[0][2] - got[1][2]) <= 512
