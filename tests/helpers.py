"""Shared test helpers: seeded graphs and fixture loading."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def fixture(name):
    return np.load(os.path.join(GOLDEN, name))


def fixture_graph(name):
    """Rebuild the graph, base vectors and queries of a traversal fixture."""
    from falcon_b200.formats import Graph
    from falcon_b200.synthetic import sift_like
    f = fixture(name)
    n, dim, nq = int(f["n"]), int(f["dim"]), int(f["n_queries"])
    x = sift_like(n, dim, seed=int(f["data_seed"]))
    q = sift_like(nq, dim, seed=int(f["query_seed"]))
    g = Graph.from_adjacency(x, f["adjacency"].astype(np.int32), int(f["entry"]))
    return f, g, q


_cache = {}


def small_graph(kind="sift", n=4000, dim=128, max_degree=32, nq=64, seed=0):
    key = (kind, n, dim, max_degree, nq, seed)
    if key not in _cache:
        from falcon_b200.graph import build_graph
        from falcon_b200.synthetic import sift_like, unit_normal
        gen = sift_like if kind == "sift" else unit_normal
        x = gen(n, dim, seed)
        q = gen(nq, dim, seed + 1)
        g = build_graph(x, max_degree, device="cpu")
        _cache[key] = (g, q)
    return _cache[key]


def oracle_graph(oracle, g, elem=0, stored=None, scales=None):
    return oracle.OracleGraph(g.vectors, g.links, g.max_degree, g.ids_offset, elem, stored, scales)
