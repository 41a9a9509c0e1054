"""Traversal trace (the reference's trace kernel,
FPGA_multi_DDR/eval_trace_FPGA_inter_query_v1.3): per expanded candidate its
distance and the number of distances computed for its row, per computed
distance the distance and the id.

CPU: the oracle's trace against the reference trace kernel itself (its HLS
sources compiled as C++ through oracle/ref_harness, built from
eval_trace_FPGA_inter_query_v1.3/src) and its internal consistency.
GPU: falcon_search_trace against the oracle, bit for bit.
"""
import numpy as np
import pytest

from helpers import oracle_graph, small_graph


def _same_trace(tr, i, cd, cn, td, ti, cnt):
    """GPU trace of query i equals the oracle's arrays (up to the capacities)."""
    c_d, c_n, d, ids = tr.query(i)
    ne, nd = len(c_d), len(d)
    return (np.array_equal(tr.counts[i], cnt[i])
            and np.array_equal(c_d.view(np.uint32), cd[i, :ne].view(np.uint32))
            and np.array_equal(c_n, cn[i, :ne])
            and np.array_equal(d.view(np.uint32), td[i, :nd].view(np.uint32))
            and np.array_equal(ids, ti[i, :nd]))


@pytest.mark.parametrize("mc,mg", [(1, 1), (2, 3), (4, 2)])
def test_oracle_trace_matches_reference_trace_kernel(oracle_mod, mc, mg):
    if not oracle_mod.ref_trace_available():
        pytest.skip("reference trace harness not built on this host")
    g, q = small_graph("sift", 2000, 128, 32, 12, seed=3)
    og = oracle_graph(oracle_mod, g)
    p = oracle_mod.make_params(k=64, ef=64, mc=mc, mg=mg)
    ids, d, hops, vis, (cd, cn, td, ti, cnt) = oracle_mod.search_trace(og, q, g.entry_point, p, 4096, 8192)
    rid, rd, rh, rv, rtr = oracle_mod.ref_inter_search_trace(g.vectors, g.links, 32, q, g.entry_point, ef=64,
                                                             mc=mc, mg=mg)
    assert np.array_equal(ids, rid) and np.array_equal(hops, rh) and np.array_equal(vis, rv)
    for i, (c_d, c_n, t_d, t_i) in enumerate(rtr):
        assert np.array_equal(cd[i, :cnt[i, 1]].view(np.uint32), c_d.view(np.uint32))
        assert np.array_equal(cn[i, :cnt[i, 1]], c_n)
        assert np.array_equal(td[i, :cnt[i, 2]].view(np.uint32), t_d.view(np.uint32))
        assert np.array_equal(ti[i, :cnt[i, 2]], t_i)


def test_oracle_trace_is_consistent(oracle_mod):
    g, q = small_graph("unit", 2000, 96, 64, 24, seed=4)
    og = oracle_graph(oracle_mod, g)
    p = oracle_mod.make_params(k=10, ef=128, mc=2, mg=2, cand_queue_size=64, bloom_bits=14)
    ids, d, hops, vis, (cd, cn, td, ti, cnt) = oracle_mod.search_trace(og, q, g.entry_point, p, 4096, 8192)
    i2, d2, h2, v2, _ = oracle_mod.search(og, q, g.entry_point, p)
    assert np.array_equal(ids, i2) and np.array_equal(hops, h2) and np.array_equal(vis, v2)
    assert np.all(cnt[:, 0] == hops) and np.all(cnt[:, 1] == hops) and np.all(cnt[:, 2] == vis)
    assert np.all(cd[:, 0] == np.float32(1e20))
    for i in range(len(q)):
        assert cn[i, :cnt[i, 1]].sum() == vis[i]
        # every traced distance is the oracle's distance of that id
        ref = oracle_mod.l2_batch(og, q[i], ti[i, :cnt[i, 2]])
        assert np.array_equal(ref.view(np.uint32), td[i, :cnt[i, 2]].view(np.uint32))
        # popped candidates come out best-first within the threshold rule: all finite after the entry
        assert np.all(cd[i, 1:cnt[i, 1]] < np.float32(1e20))


# (kind, n, dim, max_degree, k, ef, mc, mg, cq, bits): row path (degree <= 64, one register row), chunk path
# (degree > 64, wider vectors), register and bucketed result lists, global Bloom filter
CASES = [("sift", 4000, 128, 32, 10, 64, 1, 1, 32, 16),
         ("unit", 4000, 96, 64, 10, 300, 2, 3, 64, 17),
         ("unit", 3000, 384, 64, 10, 64, 2, 2, 32, 16),
         ("sift", 3000, 128, 96, 10, 128, 1, 2, 32, 15),
         ("unit", 4000, 96, 64, 10, 1024, 1, 1, 256, 20)]


@pytest.mark.gpu
@pytest.mark.parametrize("kind,n,dim,md,k,ef,mc,mg,cq,bits", CASES)
def test_gpu_trace_matches_oracle(oracle_mod, kind, n, dim, md, k, ef, mc, mg, cq, bits):
    from falcon_b200 import FalconIndex
    g, q = small_graph(kind, n, dim, md, 48, seed=11)
    ix = FalconIndex(g)
    og = oracle_graph(oracle_mod, g)
    p = dict(k=k, ef=ef, mc=mc, mg=mg, cand_queue_size=cq, bloom_bits=bits)
    ids, d, hops, vis, (cd, cn, td, ti, cnt) = oracle_mod.search_trace(og, q, g.entry_point,
                                                                       oracle_mod.make_params(**p), 4096, 16384)
    r, tr = ix.search_trace(q, cand_capacity=4096, capacity=16384, **p)
    assert np.array_equal(r.ids, ids) and np.array_equal(r.dists.view(np.uint32), d.view(np.uint32))
    assert np.array_equal(r.hops, hops) and np.array_equal(r.visited, vis)
    for i in range(len(q)):
        assert _same_trace(tr, i, cd, cn, td, ti, cnt), i
    # the traced search returns what the plain search returns
    r2 = ix.search(q, **p)
    assert np.array_equal(r2.ids, r.ids) and np.array_equal(r2.hops, r.hops)
    ix.close()


@pytest.mark.gpu
def test_gpu_trace_capacity_and_reference_streams(oracle_mod):
    """Past a capacity entries are counted, not written; the flat streams
    have the reference's -1 ... -2 framing."""
    from falcon_b200 import FalconIndex
    g, q = small_graph("sift", 4000, 128, 32, 16, seed=12)
    ix = FalconIndex(g)
    p = dict(k=10, ef=64, mc=1, mg=2)
    r, full = ix.search_trace(q, cand_capacity=4096, capacity=16384, **p)
    r2, cut = ix.search_trace(q, cand_capacity=5, capacity=40, **p)
    assert np.array_equal(full.counts, cut.counts) and np.array_equal(r.ids, r2.ids)
    assert np.array_equal(cut.cand_d, full.cand_d[:, :5]) and np.array_equal(cut.ids, full.ids[:, :40])
    cds, cns, ds, ids = full.reference_streams()
    assert cds[0] == -1 and cds[-1] == -2 and (cns == -2).sum() == len(q) and (ids == -1).sum() == len(q)
    assert len(ds) == int(full.counts[:, 2].sum()) + 2 * len(q)
    if oracle_mod.ref_trace_available():
        og = oracle_graph(oracle_mod, g)
        rid, rd, rh, rv, rtr = oracle_mod.ref_inter_search_trace(g.vectors, g.links, 32, q, g.entry_point, ef=64,
                                                                 mc=1, mg=2)
        flat = np.concatenate([np.concatenate([[-1], t[3], [-2]]) for t in rtr]).astype(np.int32)
        assert np.array_equal(flat, ids)
    ix.close()


@pytest.mark.gpu
def test_gpu_trace_device_memory_and_errors():
    """Device-memory trace buffers give the host-memory result; FP8, intra
    mode and rerank are refused."""
    import ctypes
    import torch
    from falcon_b200 import FalconIndex, _lib, make_params
    g, q = small_graph("unit", 4000, 96, 64, 16, seed=13)
    ix = FalconIndex(g)
    r, tr = ix.search_trace(q, cand_capacity=256, capacity=4096, k=10, ef=64)
    dq = torch.from_numpy(q).cuda()
    nq = len(q)
    t = lambda shape, dt: torch.zeros(shape, dtype=dt, device="cuda")
    oi, od, h, v = t((nq, 10), torch.int32), t((nq, 10), torch.float32), t(nq, torch.int32), t(nq, torch.int32)
    cd, cn, td, ti, cnt = (t((nq, 256), torch.float32), t((nq, 256), torch.int32), t((nq, 4096), torch.float32),
                           t((nq, 4096), torch.int32), t((nq, 3), torch.int32))
    prm = make_params(k=10, ef=64)
    lib = _lib.load()
    rc = lib.falcon_search_trace(ix._h, dq.data_ptr(), nq, 96, None, ctypes.byref(prm), oi.data_ptr(), od.data_ptr(),
                                 10, h.data_ptr(), v.data_ptr(), cd.data_ptr(), cn.data_ptr(), 256, td.data_ptr(),
                                 ti.data_ptr(), 4096, cnt.data_ptr(), _lib.MEM_DEVICE, None)
    _lib.check(rc)
    torch.cuda.synchronize()
    assert np.array_equal(oi.cpu().numpy(), r.ids) and np.array_equal(cnt.cpu().numpy(), tr.counts)
    from falcon_b200.index import Trace
    dev = Trace(cd.cpu().numpy(), cn.cpu().numpy(), td.cpu().numpy(), ti.cpu().numpy(), cnt.cpu().numpy())
    for i in range(nq):   # entries past the counts are unspecified: compare what was written
        for a, b in zip(dev.query(i), tr.query(i)):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    for bad in (make_params(k=10, ef=64, mode="intra", channels=4), make_params(k=10, ef=64, precision="fp8")):
        rc = lib.falcon_search_trace(ix._h, q.ctypes.data, nq, 96, None, ctypes.byref(bad), oi.data_ptr(),
                                     od.data_ptr(), 10, None, None, None, None, 0, None, None, 0,
                                     np.zeros((nq, 3), np.int32).ctypes.data, _lib.MEM_HOST, None)
        assert rc == _lib.FALCON_ERR_UNSUPPORTED
    ix.close()
