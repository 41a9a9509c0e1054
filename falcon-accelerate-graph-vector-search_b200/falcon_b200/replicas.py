"""Multi-GPU: query-sharded index replicas.

Queries are independent, so N GPUs hold N full replicas of the index (each
rank builds or loads its own) and split the query batch into contiguous
slices; the search itself has no collective.  Results come back to every
rank with one all-gather at the end (host tensors, so it works over gloo as
well as NCCL).  This mirrors the reference's inter-query channel replication
(FPGA_multi_DDR/FPGA_inter_query_v1.3_longer_FIFO_alt_PR/src/host.cpp:237-278,
DRAM_utils.hpp:54-116) one level up: GPUs instead of DDR channels.
"""
import numpy as np


def shard_bounds(n, world, rank):
    """Contiguous [start, end) slice of n items for `rank` of `world` (sizes differ by at most 1)."""
    base, rem = divmod(n, world)
    start = rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


def search_sharded(index, queries, group=None, **params):
    """Search this rank's slice of `queries` on its replica, then all-gather the
    rows so every rank holds the full (ids, dists, hops, visited)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = len(queries)
    s, e = shard_bounds(n, world, rank)
    r = index.search(np.ascontiguousarray(queries[s:e]), **params)
    ids, dists, hops, vis = (np.asarray(a) for a in (r.ids, r.dists, r.hops, r.visited))
    width = ids.shape[1] if ids.ndim == 2 and ids.shape[0] else int(params.get("k", 10))
    counts = [shard_bounds(n, world, i)[1] - shard_bounds(n, world, i)[0] for i in range(world)]
    mx = max(counts)

    def gather(a, cols, dtype):
        buf = torch.zeros((mx, cols), dtype=dtype)
        if len(a):
            buf[:len(a)] = torch.from_numpy(np.asarray(a).reshape(len(a), cols))
        out = [torch.zeros_like(buf) for _ in range(world)]
        dist.all_gather(out, buf, group=group)
        return np.concatenate([o[:c].numpy() for o, c in zip(out, counts)])

    return (gather(ids, width, torch.int32), gather(dists, width, torch.float32),
            gather(hops, 1, torch.int32)[:, 0], gather(vis, 1, torch.int32)[:, 0])


def max_over_ranks(value, group=None):
    """Max of a host scalar over all ranks (the timing rule for multi-GPU numbers)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
