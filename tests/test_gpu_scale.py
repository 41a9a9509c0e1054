"""GPU parity at the scales and operating points the benchmark runs.

* the sift100k_hnsw_m16 workload in full: the 100k x 128 base with the HNSW graph the
  reference's own scripts would build (the vendored hnswlib, M=16,
  ef_construction=128, random_seed 0, points added in order on one thread;
  vector_search_baselines/scripts_hnsw/construct_and_search_hnsw.py:124-153),
  1000 queries, k=10, ef=64, mc=1: bit-exact against the oracle (ids,
  distance bits, hops, visited), and recall@10 within 0.002 of hnswlib's own
  search on the same graph at the same ef (FPGA semantics with a candidate
  queue and filter large enough not to bind, which is what hnswlib's
  unbounded candidate heap and exact visited list amount to).
* the throughput point of the 1M x 96 workload on a 200k-node graph with
  HNSW upper layers: ef=1024, candidate queue 256, 2^19-bit filters in
  global memory, entries from the upper-layer descent, FP32 and BF16 +
  FP32 rerank: bit-exact against the oracle on 100 queries.
"""
import numpy as np
import pytest

from helpers import oracle_graph

pytestmark = pytest.mark.gpu


def _same(a_ids, a_d, b_ids, b_d):
    return np.array_equal(a_ids, b_ids) and np.array_equal(np.asarray(a_d).view(np.uint32),
                                                           np.asarray(b_d).view(np.uint32))


@pytest.fixture(scope="module")
def sift100k(oracle_mod):
    if not oracle_mod.Hnsw.available():
        pytest.skip("reference-derived hnswlib library not built on this host")
    from falcon_b200.formats import Graph, UpperLayers
    from falcon_b200.synthetic import sift_like
    x = sift_like(100_000, 128, seed=0)
    q = sift_like(1000, 128, seed=1)
    h = oracle_mod.Hnsw.build(x, 16, 128, 0)
    links, counts, labels, entry, max_level = h.level0()
    adj = np.where(np.arange(links.shape[1])[None, :] < counts[:, None], links, -1).astype(np.int32)
    ml, ep, mm, levels, starts, rows = h.upper()
    g = Graph.from_adjacency(x, adj, entry, labels)
    upper = UpperLayers(ml, mm, ep, levels, starts, rows)
    return h, g, upper, x, q


def test_sift100k_hnswlib_graph_bit_exact(sift100k, oracle_mod):
    from falcon_b200 import FalconIndex
    h, g, upper, x, q = sift100k
    assert g.max_degree == 32
    ix = FalconIndex(g)
    # the reference's multi-DDR host starts every query at the global entry (host.cpp:711-713)
    r = ix.search(q, k=10, ef=64, mc=1, mg=1, cand_queue_size=32, bloom_bits=16)
    og = oracle_graph(oracle_mod, g)
    ids, d, hops, vis, _ = oracle_mod.search(og, q, g.entry_point, oracle_mod.make_params(k=10, ef=64, mc=1, mg=1))
    # the GPU returns labels, the oracle physical ids
    assert _same(r.ids, r.dists, np.where(ids >= 0, g.labels[np.maximum(ids, 0)], -1), d)
    assert np.array_equal(r.hops, hops) and np.array_equal(r.visited, vis)
    ix.close()


def test_sift100k_recall_within_hnswlib_tolerance(sift100k):
    from falcon_b200 import FalconIndex
    from falcon_b200.groundtruth import brute_force_f64, recall_at_k
    h, g, upper, x, q = sift100k
    gt, _ = brute_force_f64(x, q, 10)
    ix = FalconIndex(g)
    ix.set_upper_layers(upper)
    for ef in (64, 128):
        lab, _ = h.search(q, 10, ef, 8)
        ours = ix.search(q, k=10, ef=ef, mc=1, mg=1, cand_queue_size=256, bloom_bits=22)
        r_ref, r_ours = recall_at_k(lab, gt, 10), recall_at_k(ours.ids, gt, 10)
        assert abs(r_ours - r_ref) <= 0.002, (ef, r_ours, r_ref)
    ix.close()


@pytest.fixture(scope="module")
def big_upper():
    from falcon_b200 import FalconIndex
    from falcon_b200.graph import build_graph, build_upper_layers
    from falcon_b200.synthetic import unit_normal
    x = unit_normal(200_000, 96, seed=61)
    q = unit_normal(100, 96, seed=62)
    g = build_graph(x, 64, device="cuda")
    upper = build_upper_layers(x, 32, seed=0, device="cuda")
    ix = FalconIndex(g, storage=("f32", "bf16"))
    ix.set_upper_layers(upper)
    return ix, g, upper, q


@pytest.mark.parametrize("prec", ["f32", "bf16"])
def test_throughput_point_at_scale_bit_exact(big_upper, oracle_mod, prec):
    ix, g, upper, q = big_upper
    P = dict(k=10, ef=1024, mc=1, mg=1, cand_queue_size=256, bloom_bits=19)
    ent, _ = ix.descend(q)
    oent, _ = oracle_mod.descend(oracle_graph(oracle_mod, g), upper, q)
    assert np.array_equal(ent, oent)
    if prec == "f32":
        r = ix.search(q, **P)
        og = oracle_graph(oracle_mod, g)
        ids, d, hops, vis, _ = oracle_mod.search(og, q, oent, oracle_mod.make_params(**P))
    else:
        r = ix.search(q, precision="bf16", rerank=True, **P)
        og = oracle_graph(oracle_mod, g, elem=oracle_mod.BF16, stored=ix.storage("bf16"))
        ids, d, hops, vis, _ = oracle_mod.search(og, q, oent, oracle_mod.make_params(rerank=True, **P))
    assert _same(r.ids, r.dists, ids, d)
    assert np.array_equal(r.hops, hops) and np.array_equal(r.visited, vis)
