"""CPU, world size 2 over gloo: the replica helpers shard a query batch, each
rank searches its slice, and the all-gathered rows equal one search of the
whole batch.  The per-rank search here is the oracle standing in for a GPU
replica (the helpers only see an object with .search)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import oracle_graph, small_graph


def test_shard_bounds_cover_exactly():
    from falcon_b200.replicas import shard_bounds
    for n in (0, 1, 7, 100, 10001):
        for w in (1, 2, 3, 8):
            spans = [shard_bounds(n, w, r) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(e - s for s, e in spans) - min(e - s for s, e in spans) <= 1


class _OracleReplica:
    def __init__(self, oracle, og, entry):
        self.oracle, self.og, self.entry = oracle, og, entry

    def search(self, q, k=10, ef=64, mc=1, mg=1):
        class R:
            pass
        r = R()
        r.ids, r.dists, r.hops, r.visited, _ = self.oracle.search(self.og, q, self.entry,
                                                                   self.oracle.make_params(k=k, ef=ef, mc=mc, mg=mg))
        return r


def _worker(rank, world, port, result_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(here)
    for p in (here, os.path.join(repo, "falcon-accelerate-graph-vector-search_b200"), os.path.join(repo, "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import oracle
    from falcon_b200.replicas import max_over_ranks, search_sharded
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    g, q = small_graph("sift", 2000, 128, 32, 37, seed=3)
    rep = _OracleReplica(oracle, oracle_graph(oracle, g), g.entry_point)
    ids, d, hops, vis = search_sharded(rep, q, k=10, ef=64, mg=2)
    t = max_over_ranks(float(rank + 1))
    if rank == 0:
        np.savez(os.path.join(result_dir, "r.npz"), ids=ids, d=d, hops=hops, vis=vis, t=t)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_sharded_search_equals_single(tmp_path, oracle_mod):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = np.load(tmp_path / "r.npz")
    g, q = small_graph("sift", 2000, 128, 32, 37, seed=3)
    ids, d, hops, vis, _ = oracle_mod.search(oracle_graph(oracle_mod, g), q, g.entry_point,
                                             oracle_mod.make_params(k=10, ef=64, mg=2))
    assert np.array_equal(res["ids"], ids) and np.array_equal(res["d"], d)
    assert np.array_equal(res["hops"], hops) and np.array_equal(res["vis"], vis)
    assert float(res["t"]) == 2.0
