"""HNSW upper layers: the hnswlib save-file reader, the reference FPGA
upper-link files, the greedy upper-layer descent, and searches that start from
the descent's entry point.

CPU tests pin the reader against hnswlib itself (the reference's vendored
hnswlib, hnswalg.h:588-616, read back through its own accessors) and the
oracle's descent against hnswlib's (hnswalg.h:514-541).  GPU tests check the
CUDA descent and the search that follows it against the oracle bit for bit.
"""
import os

import numpy as np
import pytest

from helpers import oracle_graph


def _hnsw_case(n=3000, dim=32, M=8, efc=64, seed=0):
    from falcon_b200.synthetic import unit_normal
    x = unit_normal(n, dim, seed)
    q = unit_normal(200, dim, seed + 1)
    return x, q, M, efc


@pytest.fixture(scope="module")
def hnswlib_index(tmp_path_factory, oracle_mod):
    if not oracle_mod.Hnsw.available():
        pytest.skip("reference-derived hnswlib library not built on this host")
    x, q, M, efc = _hnsw_case()
    h = oracle_mod.Hnsw.build(x, M, efc, 0)
    path = str(tmp_path_factory.mktemp("hnsw") / "index.bin")
    h.save(path)
    return h, path, x, q, M


def test_reader_matches_hnswlib(hnswlib_index):
    from falcon_b200.formats import read_hnswlib_index
    h, path, x, q, M = hnswlib_index
    g, upper, info = read_hnswlib_index(path)
    links, counts, labels, entry, max_level = h.level0()
    assert np.array_equal(g.vectors, x)
    assert np.array_equal(g.adjacency(), np.where(np.arange(links.shape[1])[None, :] < counts[:, None], links, -1))
    assert np.array_equal(g.labels, labels)
    assert g.entry_point == entry and info["maxlevel"] == max_level and info["M"] == M and info["dim"] == x.shape[1]
    ml, ep, mm, levels, starts, rows = h.upper()
    assert upper.max_level == ml and upper.entry == ep and upper.max_degree == mm
    assert np.array_equal(upper.levels, levels)
    assert np.array_equal(upper.row_start, starts)
    assert np.array_equal(upper.rows[:rows.shape[0]], rows)


def test_writer_round_trip(hnswlib_index, tmp_path):
    from falcon_b200.formats import read_hnswlib_index, write_hnswlib_index
    _, path, _, _, M = hnswlib_index
    g, upper, info = read_hnswlib_index(path)
    out = str(tmp_path / "copy.bin")
    write_hnswlib_index(out, g, upper, M=M, ef_construction=info["ef_construction"])
    g2, upper2, info2 = read_hnswlib_index(out)
    assert os.path.getsize(out) == os.path.getsize(path)
    assert np.array_equal(g2.adjacency(), g.adjacency()) and np.array_equal(g2.vectors, g.vectors)
    assert np.array_equal(g2.labels, g.labels) and g2.entry_point == g.entry_point
    for a in ("levels", "row_start", "rows"):
        assert np.array_equal(getattr(upper2, a), getattr(upper, a))
    assert {k: info2[k] for k in info if k != "max_elements"} == {k: info[k] for k in info if k != "max_elements"}


def test_fpga_upper_files_round_trip(hnswlib_index, tmp_path):
    """upper_links.bin / upper_links_pointers.bin (hnsw.py:345-373) and meta.bin."""
    from falcon_b200.formats import read_fpga_index, read_fpga_upper, read_hnswlib_index, write_fpga_index
    _, path, x, _, M = hnswlib_index
    g, upper, _ = read_hnswlib_index(path)
    d = str(tmp_path / "fpga")
    write_fpga_index(d, g, "HNSW", upper=upper)
    meta = np.fromfile(os.path.join(d, "meta.bin"), dtype=np.int32)
    assert list(meta) == [g.n, upper.max_level, upper.entry, upper.max_degree, g.max_degree]
    assert os.path.getsize(os.path.join(d, "upper_links_pointers.bin")) == 8 * g.n
    u2 = read_fpga_upper(d)
    assert np.array_equal(u2.levels, upper.levels) and u2.entry == upper.entry and u2.max_level == upper.max_level
    for v in np.nonzero(upper.levels)[0]:
        for lvl in range(1, upper.levels[v] + 1):
            assert np.array_equal(u2.row(v, lvl), upper.row(v, lvl))
    g2 = read_fpga_index(d, "HNSW", x.shape[1])
    assert np.array_equal(g2.adjacency(), g.adjacency())


def test_oracle_descent_matches_hnswlib(hnswlib_index, oracle_mod):
    """Same walk; hnswlib sums in its own (SIMD) order, the oracle in the
    adder-tree order, so a near-tie could differ: allow 1 %."""
    from falcon_b200.formats import read_hnswlib_index
    h, path, x, q, _ = hnswlib_index
    g, upper, _ = read_hnswlib_index(path)
    ent, hops = oracle_mod.descend(oracle_graph(oracle_mod, g), upper, q)
    ref = h.descend(q)
    assert (ent == ref).mean() >= 0.99
    assert np.all(hops >= upper.max_level)


def _scan_one_warp(d, cur_d, bs):
    """The one-warp descent's row scan (descend_kernel): batches of bs slots in
    order; a batch's smallest distance (first slot among equals) replaces the
    best only if strictly smaller.  Returns the chosen slot or -1."""
    best, bestd = -1, cur_d
    for b0 in range(0, len(d), bs):
        blk = d[b0:b0 + bs]
        m = blk.min()
        if m < bestd:
            bestd, best = m, b0 + int(np.argmax(blk == m))
    return best


def _scan_four_warps(d, cur_d, bs):
    """descend_block_kernel's row scan: warp w takes batches w, w+4, ...; each
    warp keeps (smallest distance bits, first slot); the block takes the
    lexicographic minimum of the four pairs and moves iff it is below cur_d."""
    bits = d.astype(np.float32).view(np.uint32).astype(np.uint64)
    keys = []
    for w in range(4):
        mb, ms = 0xFFFFFFFF, 0x7FFFFFFF
        for b0 in range(w * bs, len(d), 4 * bs):
            blk = bits[b0:b0 + bs]
            m = int(blk.min())
            if m < mb:
                mb, ms = m, b0 + int(np.argmax(blk == m))
        keys.append((mb << 32) | ms)
    k = min(keys)
    mb = k >> 32
    if mb == 0xFFFFFFFF or not (np.uint32(mb).view(np.float32) < np.float32(cur_d)):
        return -1
    return int(k & 0xFFFFFFFF)


def test_block_descent_scan_equals_one_warp_scan():
    """The four-warp split of a row scan picks the same neighbour as the
    one-warp scan: the first slot holding the row's smallest distance, if
    that distance is below the current one (tie-heavy rows, any row length)."""
    rng = np.random.default_rng(5)
    for trial in range(3000):
        n = int(rng.integers(0, 130))
        bs = int(rng.choice([4, 8, 16, 32]))
        d = rng.integers(0, 12, n).astype(np.float32) / 4.0   # few distinct values: many ties
        cur = np.float32(rng.integers(0, 14) / 4.0)
        assert _scan_four_warps(d, cur, bs) == _scan_one_warp(d, cur, bs), (trial, n, bs)


def test_synthetic_upper_layers_are_consistent():
    from falcon_b200.graph import build_upper_layers
    from falcon_b200.synthetic import unit_normal
    x = unit_normal(4000, 24, 3)
    up = build_upper_layers(x, 8, seed=2, device="cpu")
    assert up.max_level >= 1 and up.levels[up.entry] == up.max_level
    frac = (up.levels >= 1).mean()
    assert 0.07 < frac < 0.2                     # P(level >= 1) = 1/M
    for v in np.nonzero(up.levels)[0]:
        for lvl in range(1, up.levels[v] + 1):
            r = up.row(v, lvl)
            assert len(r) <= 8 and np.all(up.levels[r] >= lvl) and v not in r


@pytest.mark.gpu
def test_set_upper_layers_rejects_bad_rows(lib):
    from falcon_b200 import FalconIndex
    from falcon_b200._lib import FALCON_ERR_GRAPH, FalconError
    from falcon_b200.formats import UpperLayers
    from helpers import small_graph
    g, _ = small_graph("unit", 2000, 96, 64, 4, seed=5)
    ix = FalconIndex(g)
    lists = [[] for _ in range(g.n)]
    lists[3] = [np.array([7], dtype=np.int32)]      # 7 is not on level 1
    lists[9] = [np.array([3], dtype=np.int32)]
    with pytest.raises(FalconError) as e:
        ix.set_upper_layers(UpperLayers.from_lists(4, 3, lists))
    assert e.value.code == FALCON_ERR_GRAPH
    ix.close()


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

def _gpu_case(oracle_mod, hnswlib_path=None):
    from falcon_b200.formats import read_hnswlib_index
    from falcon_b200.graph import build_graph, build_upper_layers
    from falcon_b200.synthetic import unit_normal
    if hnswlib_path:
        g, upper, _ = read_hnswlib_index(hnswlib_path)
        q = unit_normal(200, g.dim, 1)
    else:
        x = unit_normal(6000, 96, 21)
        q = unit_normal(200, 96, 22)
        g = build_graph(x, 64, device="cuda")
        upper = build_upper_layers(x, 32, seed=4, device="cuda")
        g.entry_point = upper.entry
    return g, upper, q


@pytest.mark.gpu
@pytest.mark.parametrize("source", ["hnswlib", "synthetic"])
def test_gpu_descent_matches_oracle(oracle_mod, source, tmp_path):
    from falcon_b200 import FalconIndex
    path = None
    if source == "hnswlib":
        if not oracle_mod.Hnsw.available():
            pytest.skip("reference-derived hnswlib library not built")
        x, q, M, efc = _hnsw_case()
        h = oracle_mod.Hnsw.build(x, M, efc, 0)
        path = str(tmp_path / "index.bin")
        h.save(path)
    g, upper, q = _gpu_case(oracle_mod, path)
    ix = FalconIndex(g)
    ix.set_upper_layers(upper)
    ent, hops = ix.descend(q)
    oent, ohops = oracle_mod.descend(oracle_graph(oracle_mod, g), upper, q)
    assert np.array_equal(ent, oent) and np.array_equal(hops, ohops)
    import torch
    dent, dhops = ix.descend(torch.from_numpy(q).cuda())
    assert np.array_equal(dent.cpu().numpy(), oent) and np.array_equal(dhops.cpu().numpy(), ohops)
    # small batches run a block per query, large ones a warp per query: both
    # kernels (1000 queries here, the 200 above tiled) give the oracle's entries
    big = np.tile(q, (5, 1))
    bent, bhops = ix.descend(big)
    assert np.array_equal(bent, np.tile(oent, 5)) and np.array_equal(bhops, np.tile(ohops, 5))
    ent1, hops1 = ix.descend(q[:1])
    assert ent1[0] == oent[0] and hops1[0] == ohops[0]
    ix.close()


@pytest.mark.gpu
def test_gpu_search_starts_from_descent(oracle_mod):
    """Without entry points an index with upper layers searches from the
    descent's entry: identical to the oracle searching from the oracle's
    descent, through falcon_search (host and device memory) and
    falcon_search_noalloc."""
    import ctypes
    import torch
    from falcon_b200 import FalconIndex, _lib, make_params
    g, upper, q = _gpu_case(oracle_mod)
    ix = FalconIndex(g)
    ix.set_upper_layers(upper)
    og = oracle_graph(oracle_mod, g)
    oent, _ = oracle_mod.descend(og, upper, q)
    p = dict(k=10, ef=128, mc=2, mg=2, cand_queue_size=64, bloom_bits=17)
    ids, d, hops, vis, _ = oracle_mod.search(og, q, oent, oracle_mod.make_params(**p))
    r = ix.search(q, **p)
    assert np.array_equal(r.ids, ids) and np.array_equal(r.dists.view(np.uint32), d.view(np.uint32))
    assert np.array_equal(r.hops, hops) and np.array_equal(r.visited, vis)
    rd = ix.search(torch.from_numpy(q).cuda(), **p)
    assert np.array_equal(rd.ids.cpu().numpy(), ids) and np.array_equal(rd.hops.cpu().numpy(), hops)
    # the no-allocation entry point takes its entries from the static scratch
    dq = torch.from_numpy(q).cuda()
    oi = torch.empty((len(q), 10), dtype=torch.int32, device="cuda")
    od = torch.empty((len(q), 10), dtype=torch.float32, device="cuda")
    prm = make_params(**p)
    rc = _lib.load().falcon_search_noalloc(ix._h, dq.data_ptr(), len(q), q.shape[1], None, ctypes.byref(prm), 0,
                                           oi.data_ptr(), od.data_ptr(), 10, None, None, None)
    _lib.check(rc)
    torch.cuda.synchronize()
    assert np.array_equal(oi.cpu().numpy(), ids)
    # explicit entry points still win over the descent
    r2 = ix.search(q, entry_points=np.full(len(q), g.entry_point, dtype=np.int32), **p)
    ids2, _, _, _, _ = oracle_mod.search(og, q, g.entry_point, oracle_mod.make_params(**p))
    assert np.array_equal(r2.ids, ids2)
    ix.close()
