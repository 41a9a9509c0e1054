"""GPU parity: the sm_100a kernels through the C ABI against the oracle.

Integer, index and queue work is compared bit for bit: returned ids, the bit
patterns of the FP32 distances, hops and visited counts.  The reduced
precision traversals (BF16, FP8 + per-vector scale) are compared bit for bit
too: the oracle decodes the very codes the index stores and runs the same
adder tree.
"""
import numpy as np
import pytest

from helpers import fixture_graph, oracle_graph, small_graph

pytestmark = pytest.mark.gpu


def _index(g, storage=("f32",)):
    from falcon_b200 import FalconIndex
    return FalconIndex(g, storage=storage)


def _same(a_ids, a_d, b_ids, b_d):
    return np.array_equal(a_ids, b_ids) and np.array_equal(np.asarray(a_d).view(np.uint32),
                                                           np.asarray(b_d).view(np.uint32))


@pytest.mark.parametrize("name", ["traversal_d128_md32.npz", "traversal_d96_md64.npz"])
def test_gpu_matches_reference_fixture(name):
    f, g, q = fixture_graph(name)
    ix = _index(g)
    for i, (ef, mc, mg, cq, bits) in enumerate(f["params"]):
        r = ix.search(q, k=int(ef), ef=int(ef), mc=int(mc), mg=int(mg), cand_queue_size=int(cq), bloom_bits=int(bits))
        assert _same(r.ids, r.dists, f["ids_%d" % i], f["dists_%d" % i]), (name, i)
        assert np.array_equal(r.hops, f["hops_%d" % i])
        assert np.array_equal(r.visited, f["visited_%d" % i])


CASES = [
    # kind, n, dim, md, k, ef, mc, mg, cq, bits
    ("sift", 6000, 128, 32, 10, 64, 1, 1, 32, 16),
    ("sift", 6000, 128, 32, 10, 64, 1, 4, 32, 16),
    ("sift", 6000, 128, 32, 64, 64, 2, 3, 32, 16),
    ("sift", 6000, 128, 32, 1, 10, 1, 2, 8, 10),
    ("sift", 6000, 128, 32, 100, 256, 4, 8, 32, 18),
    ("unit", 6000, 96, 64, 10, 64, 1, 1, 32, 16),
    ("unit", 6000, 96, 64, 10, 128, 2, 6, 32, 16),
    ("unit", 6000, 96, 64, 32, 200, 8, 2, 32, 17),
    ("unit", 4000, 384, 64, 10, 64, 2, 2, 32, 16),
    ("unit", 4000, 200, 48, 10, 96, 3, 16, 24, 14),
    ("sift", 4000, 50, 20, 5, 33, 1, 5, 31, 13),
    # vectors of <= 16 segments share a register row with others (lane groups)
    ("sift", 4000, 32, 32, 10, 128, 2, 2, 32, 15),
    ("unit", 6000, 64, 64, 10, 600, 1, 2, 128, 20),
    # beyond the reference hardware's ef <= 64 and 32-entry candidate queue
    ("unit", 6000, 96, 64, 10, 512, 1, 2, 64, 16),
    ("unit", 6000, 96, 64, 10, 1024, 2, 4, 256, 17),
    ("sift", 6000, 128, 32, 50, 300, 4, 3, 100, 16),
    ("unit", 4000, 384, 64, 10, 700, 1, 1, 128, 16),
    # Bloom filters above 2^18 bits live in global memory
    ("unit", 6000, 96, 64, 10, 256, 2, 2, 64, 20),
    ("sift", 6000, 128, 32, 10, 1024, 1, 3, 256, 22),
]


@pytest.mark.parametrize("kind,n,dim,md,k,ef,mc,mg,cq,bits", CASES)
def test_gpu_matches_oracle_f32(oracle_mod, kind, n, dim, md, k, ef, mc, mg, cq, bits):
    g, q = small_graph(kind, n, dim, md, 96, seed=7)
    ix = _index(g)
    r = ix.search(q, k=k, ef=ef, mc=mc, mg=mg, cand_queue_size=cq, bloom_bits=bits)
    og = oracle_graph(oracle_mod, g)
    ids, d, hops, vis, _ = oracle_mod.search(og, q, g.entry_point, oracle_mod.make_params(
        k=k, ef=ef, mc=mc, mg=mg, cand_queue_size=cq, bloom_bits=bits))
    assert _same(r.ids, r.dists, ids, d)
    assert np.array_equal(r.hops, hops)
    assert np.array_equal(r.visited, vis)


# (precision, dim, rerank, ef, mc, mg, cand_queue_size, bloom_bits).  Vectors of
# at most 16 segments are packed several to a register row of the warp
# (bf16 dim <= 128, fp8 dim <= 256, f32 dim <= 64), larger ones are not.
RP_CASES = [("bf16", 128, False, 64, 2, 2, 32, 16), ("bf16", 384, True, 64, 2, 2, 32, 16),
            ("fp8", 96, False, 64, 2, 2, 32, 16), ("fp8", 384, True, 64, 2, 2, 32, 16),
            ("bf16", 96, True, 64, 2, 2, 32, 16), ("fp8", 32, False, 100, 1, 3, 48, 15),
            ("bf16", 48, True, 200, 4, 2, 64, 16), ("bf16", 96, True, 1024, 1, 1, 256, 20),
            ("fp8", 96, True, 512, 2, 2, 128, 19)]


@pytest.mark.parametrize("prec,dim,rerank,ef,mc,mg,cq,bits", RP_CASES)
def test_gpu_reduced_precision_matches_oracle(oracle_mod, prec, dim, rerank, ef, mc, mg, cq, bits):
    g, q = small_graph("unit", 4000, dim, 64, 64, seed=9)
    ix = _index(g, storage=("f32", prec))
    r = ix.search(q, k=10, ef=ef, mc=mc, mg=mg, cand_queue_size=cq, bloom_bits=bits, precision=prec, rerank=rerank)
    if prec == "bf16":
        codes, scales, elem = ix.storage("bf16"), None, oracle_mod.BF16
    else:
        (codes, scales), elem = ix.storage("fp8"), oracle_mod.FP8
    og = oracle_graph(oracle_mod, g, elem=elem, stored=codes, scales=scales)
    ids, d, hops, vis, _ = oracle_mod.search(og, q, g.entry_point, oracle_mod.make_params(
        k=10, ef=ef, mc=mc, mg=mg, cand_queue_size=cq, bloom_bits=bits, rerank=rerank))
    assert _same(r.ids, r.dists, ids, d)
    assert np.array_equal(r.hops, hops) and np.array_equal(r.visited, vis)


def test_encoders_match_host_rounding():
    g, _ = small_graph("unit", 4000, 96, 64, 4, seed=9)
    ix = _index(g, storage=("f32", "bf16", "fp8"))
    f32 = ix.storage("f32")
    assert np.array_equal(f32[:, :96], g.vectors) and np.all(f32[:, 96:] == 0)
    bf = ix.storage("bf16").astype(np.uint32)
    u = g.vectors.view(np.uint32)
    rne = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16)          # round-to-nearest-even to bf16
    assert np.array_equal(bf[:, :96], rne)
    codes, scales = ix.storage("fp8")
    amax = np.abs(g.vectors).max(1)
    assert np.array_equal(scales, (amax / np.float32(448.0)).astype(np.float32))
    import oracle
    table = np.array([oracle.fp8_to_f32(c) for c in range(256)], dtype=np.float32)
    dec = table[codes[:, :96]] * scales[:, None]
    err = np.abs(dec - g.vectors) / amax[:, None]
    assert err.max() <= 2.0 ** -4 * 1.01                     # half an E4M3 ulp at the top binade


def test_mixed_per_query_params_one_launch(oracle_mod):
    g, q = small_graph("sift", 6000, 128, 32, 96, seed=7)
    rng = np.random.default_rng(5)
    pq = []
    for _ in range(len(q)):
        pq.append(dict(k=int(rng.choice([1, 10, 100])), ef=int(rng.choice([32, 64, 128, 256])),
                       mc=int(rng.choice([1, 2, 4])), mg=int(rng.integers(1, 6))))
    ix = _index(g)
    r = ix.search(q, per_query=pq)
    og = oracle_graph(oracle_mod, g)
    ps = [oracle_mod.make_params(**p) for p in pq]
    ids, d, hops, vis, _ = oracle_mod.search(og, q, g.entry_point, ps, out_stride=r.ids.shape[1])
    assert _same(r.ids, r.dists, ids, d)
    assert np.array_equal(r.hops, hops) and np.array_equal(r.visited, vis)
    for i, p in enumerate(pq):
        assert np.all(r.ids[i, max(p["k"], 1):] == -1) or p["k"] == r.ids.shape[1]


def test_vadd_dropin_matches_fixture():
    from falcon_b200 import vadd
    from falcon_b200.formats import reference_vector_rows, pad16
    f, g, q = fixture_graph("traversal_d128_md32.npz")
    qp = np.zeros((len(q), pad16(128)), dtype=np.float32)
    qp[:] = q
    ef, mc, mg, cq, bits = [int(v) for v in f["params"][1]]
    oid, od, dbg = vadd(qp, np.full(len(q), g.entry_point, np.int32), reference_vector_rows(g.vectors), g.links,
                        g.n, 128, ef=ef, candidate_queue_runtime_size=cq, max_cand_batch_size=mc,
                        max_async_stage_num=mg, runtime_n_bucket_addr_bits=bits, max_link_num_base=32)
    assert _same(oid, od, f["ids_1"], f["dists_1"])
    assert np.array_equal(dbg[:, 0], f["hops_1"]) and np.array_equal(dbg[:, 1], f["visited_1"])


def test_load_fpga_files_and_labels(tmp_path):
    from falcon_b200 import FalconIndex
    from falcon_b200.formats import Graph, write_fpga_index
    g, q = small_graph("sift", 6000, 128, 32, 32, seed=7)
    labels = (np.arange(g.n, dtype=np.int32) * 7 + 3)
    gl = Graph(g.vectors, g.links, g.max_degree, g.entry_point, labels)
    write_fpga_index(str(tmp_path / "h"), gl, "HNSW")
    write_fpga_index(str(tmp_path / "n"), g, "NSG")
    mem = _index(g).search(q, k=10, ef=64)
    h = FalconIndex.load_fpga(str(tmp_path / "h"), "HNSW", 128).search(q, k=10, ef=64)
    n = FalconIndex.load_fpga(str(tmp_path / "n"), "NSG", 128).search(q, k=10, ef=64)
    assert _same(n.ids, n.dists, mem.ids, mem.dists)
    assert np.array_equal(h.ids, np.where(mem.ids >= 0, mem.ids * 7 + 3, -1))
    assert np.array_equal(h.hops, mem.hops)


def test_load_multichannel_fpga_files(tmp_path):
    """A directory holding only the 4-channel set (the layout of the
    reference's 4-channel FPGA builds) loads and searches like the graph."""
    from falcon_b200 import FalconIndex
    from falcon_b200.formats import write_fpga_index
    g, q = small_graph("sift", 6001, 128, 32, 32, seed=9)
    write_fpga_index(str(tmp_path / "n4"), g, "NSG", num_channels=(4,))
    mem = _index(g).search(q, k=10, ef=64, mc=2, mg=2)
    r = FalconIndex.load_fpga(str(tmp_path / "n4"), "NSG", 128).search(q, k=10, ef=64, mc=2, mg=2)
    assert _same(r.ids, r.dists, mem.ids, mem.dists)
    assert np.array_equal(r.hops, mem.hops) and np.array_equal(r.visited, mem.visited)


def test_device_memory_path_matches_host():
    import torch
    g, q = small_graph("unit", 6000, 96, 64, 96, seed=7)
    ix = _index(g)
    h = ix.search(q, k=10, ef=64, mc=2, mg=3)
    dq = torch.from_numpy(q).cuda()
    d = ix.search(dq, k=10, ef=64, mc=2, mg=3)
    torch.cuda.synchronize()
    assert _same(h.ids, h.dists, d.ids.cpu().numpy(), d.dists.cpu().numpy())
    assert np.array_equal(h.hops, d.hops.cpu().numpy())
    # result tensors supplied by the caller and reused across calls (one query at a time)
    from falcon_b200.index import device_results
    out = device_results(1, 10)
    for i in (0, 5, 17):
        r = ix.search(dq[i:i + 1], k=10, ef=64, mc=2, mg=3, out=out)
        assert r.ids is out[0]
        torch.cuda.synchronize()
        assert _same(h.ids[i:i + 1], h.dists[i:i + 1], out[0].cpu().numpy(), out[1].cpu().numpy())
        assert h.hops[i] == int(out[2][0]) and h.visited[i] == int(out[3][0])
    with pytest.raises(ValueError):
        ix.search(dq[:2], k=10, ef=64, out=out)


def test_max_hops_truncation_matches_oracle(oracle_mod):
    from falcon_b200 import _lib
    g, q = small_graph("sift", 6000, 128, 32, 96, seed=7)
    r = _index(g).search(q, k=10, ef=64, mg=3, max_hops=7)
    assert r.status == _lib.FALCON_WARN_TRUNCATED and r.hops.max() <= 7
    ids, d, hops, vis, rc = oracle_mod.search(oracle_graph(oracle_mod, g), q, g.entry_point,
                                              oracle_mod.make_params(k=10, ef=64, mg=3, max_hops=7))
    assert rc == 1 and _same(r.ids, r.dists, ids, d) and np.array_equal(r.hops, hops)


def test_edge_cases(oracle_mod):
    from falcon_b200 import FalconIndex, _lib
    from falcon_b200.formats import Graph
    g, q = small_graph("sift", 6000, 128, 32, 8, seed=7)
    ix = _index(g)
    # no queries
    r = ix.search(q[:0], k=10, ef=64)
    assert r.ids.shape == (0, 10)
    # k > ef raises ef to k
    a = ix.search(q, k=80, ef=64)
    b = ix.search(q, k=80, ef=80)
    assert _same(a.ids, a.dists, b.ids, b.dists)
    # entry node without neighbours: nothing is visited, results are empty slots
    adj = g.adjacency()
    adj[g.entry_point] = -1
    g0 = Graph.from_adjacency(g.vectors, adj, g.entry_point)
    r = FalconIndex(g0).search(q, k=5, ef=16)
    assert np.all(r.ids == -1) and np.all(r.dists == np.float32(1e20)) and np.all(r.hops == 1)
    assert np.all(r.visited == 0)
    # duplicate ids inside a row are visited once (Bloom) like the reference
    adj = g.adjacency()
    row = adj[g.entry_point]
    c = int((row >= 0).sum())
    row[c // 2:c] = row[0]
    gd = Graph.from_adjacency(g.vectors, adj, g.entry_point)
    r = FalconIndex(gd).search(q, k=10, ef=64)
    ids, d, hops, vis, _ = oracle_mod.search(oracle_graph(oracle_mod, gd), q, g.entry_point,
                                             oracle_mod.make_params(k=10, ef=64))
    assert _same(r.ids, r.dists, ids, d) and np.array_equal(r.visited, vis)
    # per-query entry points
    ep = (np.arange(len(q)) * 131) % g.n
    r = ix.search(q, k=10, ef=64, entry_points=ep)
    ids, d, hops, vis, _ = oracle_mod.search(oracle_graph(oracle_mod, g), q, ep, oracle_mod.make_params(k=10, ef=64))
    assert _same(r.ids, r.dists, ids, d)
    # a single-node graph
    g1 = Graph.from_adjacency(g.vectors[:1], np.full((1, 4), -1, np.int32), 0)
    r = FalconIndex(g1).search(q, k=3, ef=8)
    assert np.all(r.ids == -1)


def test_bad_parameters_are_errors():
    from falcon_b200 import _lib
    g, q = small_graph("sift", 6000, 128, 32, 8, seed=7)
    ix = _index(g)
    for kw in (dict(mc=0), dict(mc=9), dict(mg=17), dict(ef=1025), dict(cand_queue_size=257), dict(bloom_bits=9),
               dict(bloom_bits=25), dict(precision="bf16"), dict(k=0)):
        with pytest.raises(_lib.FalconError) as e:
            ix.search(q, **kw)
        assert e.value.code == _lib.FALCON_ERR_ARG, kw
    with pytest.raises(_lib.FalconError):
        ix.search(q, entry_points=np.full(len(q), g.n, np.int32))


def test_full_size_properties():
    """Size-independent checks on a large graph: every returned distance is the
    exact FP32 tree distance of its id, rows ascend, ids are unique, and the
    search finds the FP64 neighbours."""
    import oracle
    from falcon_b200.graph import build_graph
    from falcon_b200.groundtruth import shortlist_f64, recall_at_k
    from falcon_b200.synthetic import sift_like
    x = sift_like(200_000, 128, 21)
    q = sift_like(2000, 128, 22)
    g = build_graph(x, 32, device="cuda")
    r = _index(g).search(q, k=10, ef=64, mc=1, mg=4)
    og = oracle_graph(oracle, g)
    for i in range(0, len(q), 50):
        ok = r.ids[i] >= 0
        assert np.array_equal(oracle.l2_batch(og, q[i], r.ids[i][ok]).view(np.uint32), r.dists[i][ok].view(np.uint32))
    assert np.all(np.diff(r.dists, axis=1) >= 0)
    assert all(len(set(row.tolist())) == len(row) for row in r.ids)
    gt, _ = shortlist_f64(x, q, 10)
    rec64 = recall_at_k(r.ids, gt, 10)
    rec256 = recall_at_k(_index(g).search(q, k=10, ef=256, mc=1, mg=4).ids, gt, 10)
    # i.i.d. per-dimension data has full intrinsic dimension, so graph search
    # recall is modest; it must still rise with ef
    assert rec64 > 0.3 and rec256 > rec64 + 0.1
    sub = slice(0, 300)
    ids, d, hops, vis, _ = oracle.search(og, q[sub], g.entry_point, oracle.make_params(k=10, ef=64, mc=1, mg=4))
    assert _same(r.ids[sub], r.dists[sub], ids, d) and np.array_equal(r.visited[sub], vis)


INTRA_CASES = [
    # kind, dim, md, ef, mc, mg, channels, bits, precision
    ("unit", 96, 64, 64, 1, 1, 4, 16, "f32"),
    ("unit", 96, 64, 64, 2, 6, 4, 16, "f32"),
    ("unit", 96, 64, 128, 4, 3, 8, 15, "f32"),
    ("sift", 128, 32, 64, 2, 2, 2, 17, "f32"),
    ("sift", 128, 32, 32, 1, 4, 1, 16, "f32"),
    ("unit", 384, 64, 64, 2, 2, 4, 16, "bf16"),
    ("unit", 96, 64, 256, 8, 4, 4, 16, "fp8"),
    ("unit", 96, 64, 1024, 2, 2, 4, 16, "f32"),
    ("unit", 96, 64, 512, 1, 2, 4, 21, "f32"),
    ("sift", 128, 32, 256, 2, 2, 2, 20, "bf16"),
]


def test_gpu_intra_matches_reference_v15_fixture():
    """Intra-query mode against the reference's own v1.5 kernel pipeline
    (fixture made by tests/golden/make_golden.py): ids, distance bits, hops."""
    from falcon_b200.formats import Graph
    from falcon_b200.synthetic import unit_normal
    from helpers import fixture
    f = fixture("intra_v15_d96_md64.npz")
    x = unit_normal(int(f["n"]), int(f["dim"]), seed=int(f["data_seed"]))
    q = unit_normal(int(f["n_queries"]), int(f["dim"]), seed=int(f["query_seed"]))
    g = Graph.from_adjacency(x, f["adjacency"].astype(np.int32), int(f["entry"]))
    ix = _index(g)
    for i, (ch, ef, mc, mg, bits) in enumerate(f["params"]):
        r = ix.search(q, k=int(ef), ef=int(ef), mc=int(mc), mg=int(mg), bloom_bits=int(bits), mode="intra",
                      channels=int(ch))
        assert _same(r.ids, r.dists, f["ids_%d" % i], f["dists_%d" % i])
        assert np.array_equal(r.hops, f["hops_%d" % i])


@pytest.mark.parametrize("kind,dim,md,ef,mc,mg,ch,bits,prec", INTRA_CASES)
def test_gpu_intra_matches_oracle(oracle_mod, kind, dim, md, ef, mc, mg, ch, bits, prec):
    g, q = small_graph(kind, 4000, dim, md, 64, seed=13)
    ix = _index(g, storage=("f32", prec))
    cq = 256 if ef > 256 else 32
    r = ix.search(q, k=10, ef=ef, mc=mc, mg=mg, mode="intra", channels=ch, bloom_bits=bits, precision=prec,
                  cand_queue_size=cq)
    if prec == "f32":
        og = oracle_graph(oracle_mod, g)
    elif prec == "bf16":
        og = oracle_graph(oracle_mod, g, elem=oracle_mod.BF16, stored=ix.storage("bf16"))
    else:
        codes, scales = ix.storage("fp8")
        og = oracle_graph(oracle_mod, g, elem=oracle_mod.FP8, stored=codes, scales=scales)
    ids, d, hops, vis, _ = oracle_mod.search(og, q, g.entry_point, oracle_mod.make_params(
        k=10, ef=ef, mc=mc, mg=mg, mode="intra", channels=ch, bloom_bits=bits, cand_queue_size=cq))
    assert _same(r.ids, r.dists, ids, d)
    assert np.array_equal(r.hops, hops) and np.array_equal(r.visited, vis)


@pytest.mark.parametrize("ch,mc,mg", [(4, 2, 4), (2, 1, 1), (8, 1, 3)])
def test_gpu_intra_batch_layout_matches_oracle(oracle_mod, ch, mc, mg):
    """More queries than SMs: blocks of one fetch warp per channel plus the
    merge warp (the latency layout, up to 12 fetch warps, is the one the other
    intra cases run)."""
    g, q = small_graph("unit", 4000, 96, 64, 300, seed=17)
    ix = _index(g)
    r = ix.search(q, k=10, ef=128, mc=mc, mg=mg, mode="intra", channels=ch, bloom_bits=16)
    og = oracle_graph(oracle_mod, g)
    ids, d, hops, vis, _ = oracle_mod.search(og, q, g.entry_point, oracle_mod.make_params(
        k=10, ef=128, mc=mc, mg=mg, mode="intra", channels=ch, bloom_bits=16))
    assert _same(r.ids, r.dists, ids, d)
    assert np.array_equal(r.hops, hops) and np.array_equal(r.visited, vis)


def test_gpu_intra_mixed_params_and_truncation(oracle_mod):
    g, q = small_graph("unit", 4000, 96, 64, 64, seed=13)
    rng = np.random.default_rng(8)
    pq = [dict(k=int(rng.choice([1, 10, 50])), ef=int(rng.choice([32, 64, 128])), mc=int(rng.choice([1, 2, 4])),
               mg=int(rng.integers(1, 5)), mode="intra", channels=4, max_hops=int(rng.choice([0, 0, 9])))
          for _ in range(len(q))]
    r = _index(g).search(q, per_query=pq)
    ids, d, hops, vis, _ = oracle_mod.search(oracle_graph(oracle_mod, g), q, g.entry_point,
                                             [oracle_mod.make_params(**p) for p in pq], out_stride=r.ids.shape[1])
    assert _same(r.ids, r.dists, ids, d)
    assert np.array_equal(r.hops, hops) and np.array_equal(r.visited, vis)
