"""Scene sharding for the batched workload on several ranks (CPU, gloo)."""
import os
import socket

import numpy as np
import pytest

from colb_b200 import scene as S, shard


def test_partition_covers_every_scene_once_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.integers(100, 5000, size=101)
    for world in (1, 2, 3, 8):
        parts = shard.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        # LPT bound: the most loaded rank is within the largest item of the mean
        assert max(loads) <= costs.sum() / world + costs.max()
    assert shard.partition(costs, 4) == shard.partition(costs, 4)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        scenes = S.config3_batch(n_scenes=12, seed=3, nmin=2, nmax=6)
        mine, idx = shard.shard(scenes, rank, world)
        # per-scene statistic each rank computes for its own scenes: bodies, vertices
        local = [[len(sc["mass"]), len(sc["xbar"])] for sc in mine]
        full = shard.gather_stats(local, idx, len(scenes), 2)
        q.put((rank, idx, full.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_gather_with_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    scenes = S.config3_batch(n_scenes=12, seed=3, nmin=2, nmax=6)
    want = [[len(sc["mass"]), len(sc["xbar"])] for sc in scenes]
    idx = {r: i for r, i, _ in res}
    assert sorted(idx[0] + idx[1]) == list(range(12)) and not set(idx[0]) & set(idx[1])
    for _, _, full in res:
        assert np.array_equal(np.array(full), np.array(want, dtype=float))
