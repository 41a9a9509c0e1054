"""The hnswlib baseline harness (test and baseline infrastructure): an index
rebuilt from an exported graph (base layer + upper layers) searches exactly
like the index hnswlib built itself, and per-query (ef, k) grouping equals
separate calls."""
import numpy as np
import pytest

import oracle
from falcon_b200.formats import UpperLayers

pytestmark = pytest.mark.skipif(not oracle.Hnsw.available(), reason="hnswlib harness not built")


def _upper_of(h):
    ml, ep, mm, levels, starts, rows = h.upper()
    return UpperLayers(ml, mm, ep, levels, starts, rows)


def test_from_graph_with_upper_layers_equals_built_index():
    from falcon_b200.synthetic import sift_like
    x = sift_like(3000, 32, seed=9)
    q = sift_like(100, 32, seed=10)
    h = oracle.Hnsw.build(x, 8, 64, 0)
    links, counts, labels, ep, ml = h.level0()
    assert ml >= 1
    r = oracle.Hnsw.from_graph(x, links, ep)
    r.set_upper(_upper_of(h))
    for ef in (16, 64):
        a = h.search(q, 10, ef, 2)
        b = r.search(q, 10, ef, 2)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    h.free()
    r.free()


def test_search_mixed_matches_grouped_calls():
    from falcon_b200.synthetic import sift_like
    x = sift_like(2000, 16, seed=3)
    q = sift_like(60, 16, seed=4)
    h = oracle.Hnsw.build(x, 8, 32, 0)
    rng = np.random.default_rng(1)
    ks, efs = rng.choice([1, 10, 20], 60), rng.choice([16, 32], 60)
    lab, d = h.search_mixed(q, ks, efs, 2)
    for i in range(60):
        l1, d1 = h.search(q[i:i + 1], int(ks[i]), int(efs[i]), 1)
        assert np.array_equal(lab[i, :ks[i]], l1[0]) and np.array_equal(d[i, :ks[i]], d1[0])
        assert (lab[i, ks[i]:] == -1).all()
    h.free()


def test_isa_and_cpu_model_strings():
    assert oracle.Hnsw.isa() in ("avx2", "x86-64-v4")
    assert isinstance(oracle.Hnsw.cpu_model(), str)
