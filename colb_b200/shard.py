"""Scene sharding across ranks for the batched workload.

Independent scenes need no exchange inside a step, so the multi-GPU form of a
batch is a partition: every rank steps its own subset on its own GPU in one
handle, and the only collective is the final gather of per-scene statistics.
Scenes are assigned by longest-processing-time-first on their primitive count
(vertices + edges + triangles), which bounds the most loaded rank by 4/3 of the
optimum.
"""
import numpy as np


def scene_cost(sc):
    return int(len(sc["xbar"]) + len(sc["edges"]) + len(sc["tris"]))


def partition(costs, world):
    """Indices of the scenes of each rank (each list ascending)."""
    costs = np.asarray(costs, dtype=np.int64)
    order = np.lexsort((np.arange(len(costs)), -costs))     # cost descending, index ascending
    load = np.zeros(world, dtype=np.int64)
    parts = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))                              # least loaded, lowest rank on ties
        parts[r].append(int(i))
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def shard(scenes, rank, world):
    """This rank's scenes and their global indices."""
    idx = partition([scene_cost(s) for s in scenes], world)[rank]
    return [scenes[i] for i in idx], idx


def gather_stats(local, idx, n_total, width, group=None):
    """All ranks' per-scene rows (local: [len(idx)][width]) in global scene
    order, on every rank, through torch.distributed (gloo or NCCL)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    k = int(width)
    local = np.asarray(local, dtype=np.float64).reshape(len(idx), k)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    mine = torch.tensor([len(idx)], dtype=torch.int64, device=dev)
    counts = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(counts, mine, group=group)
    m = max(1, max(int(c.item()) for c in counts))
    buf = torch.full((m, k + 1), -1.0, dtype=torch.float64, device=dev)
    if len(idx):
        buf[:len(idx), 0] = torch.tensor(idx, dtype=torch.float64)
        buf[:len(idx), 1:] = torch.from_numpy(local)
    outs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    full = np.full((n_total, k), np.nan)
    for o in outs:
        o = o.cpu().numpy()
        for row in o:
            if row[0] >= 0:
                full[int(row[0])] = row[1:]
    return full
