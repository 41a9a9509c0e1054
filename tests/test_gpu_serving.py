"""GPU: the continuous-batching server.  Every request's result in the mix
(several resident indexes, mixed precision and k/ef/mc/mg, requests admitted
while others run) must equal the same request searched alone through
falcon_search: ids, distance bits, hops and visited, bit for bit."""
import time

import numpy as np
import pytest

from helpers import small_graph

pytestmark = pytest.mark.gpu


def _alone(ix, q, p):
    r = ix.search(q[None, :], **p)
    return r.ids[0, :p["k"]], r.dists[0, :p["k"]], int(r.hops[0]), int(r.visited[0])


def _same(a, b):
    return (np.array_equal(a[0], b[0]) and np.array_equal(np.asarray(a[1]).view(np.uint32),
                                                          np.asarray(b[1]).view(np.uint32))
            and a[2] == b[2] and a[3] == b[3])


@pytest.fixture(scope="module")
def two_indexes():
    from falcon_b200 import FalconIndex
    g1, q1 = small_graph("sift", 6000, 128, 32, 64, seed=31)
    g2, q2 = small_graph("unit", 4000, 384, 64, 64, seed=32)
    ix1 = FalconIndex(g1, storage=("f32",))
    ix2 = FalconIndex(g2, storage=("f32", "bf16", "fp8"))
    return (ix1, q1), (ix2, q2)


def _mixed_requests(two_indexes, n, seed):
    (ix1, q1), (ix2, q2) = two_indexes
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        which = int(rng.integers(0, 2))
        p = dict(k=int(rng.choice([1, 10, 50])), ef=int(rng.choice([32, 64, 128, 200])), mc=int(rng.choice([1, 2, 4])),
                 mg=int(rng.integers(1, 5)))
        if which == 1:
            prec = str(rng.choice(["f32", "bf16", "fp8"]))
            p.update(precision=prec, rerank=(prec != "f32" and bool(rng.integers(0, 2))))
        p["ef"] = max(p["ef"], p["k"])
        q = (q1 if which == 0 else q2)[i % 64]
        reqs.append((which, q, p))
    return reqs


def test_server_results_equal_alone(two_indexes):
    from falcon_b200.serving import FalconServer
    (ix1, _), (ix2, _) = two_indexes
    sv = FalconServer(ring_capacity=4096, max_k=50, ef_max=256, cand_queue_max=64, dim_max=384, idle_exit_us=3000)
    ids = [sv.add_index(ix1), sv.add_index(ix2)]
    reqs = _mixed_requests(two_indexes, 300, seed=1)
    rids = []
    # submit in small bursts so later requests are admitted while earlier ones run
    for s in range(0, len(reqs), 16):
        part = reqs[s:s + 16]
        for w, q, p in part:
            r = sv.submit([ids[w]], q[None, :], p)
            assert len(r) == 1
            rids.append(r[0])
    for (w, q, p), rid in zip(reqs, rids):
        got = sv.wait(rid, p["k"])
        ref = _alone(ix1 if w == 0 else ix2, q, p)
        assert _same(got, ref), (w, p)
    info = sv.info()
    assert info.in_flight == 0 and info.submitted == len(reqs)
    # the classes of the mix (FP32 at D=128 and D=384, BF16, FP8) share the GPU
    assert info.concurrent_classes_max >= 2
    sv.close()


def test_server_admission_by_ring_entries(two_indexes):
    from falcon_b200.serving import FalconServer
    (ix1, q1), _ = two_indexes
    sv = FalconServer(ring_capacity=8, max_k=10, ef_max=64, dim_max=128, idle_exit_us=2000)
    i0 = sv.add_index(ix1)
    p = dict(k=10, ef=64)
    r = sv.submit(np.full(20, i0), q1[:20], p)
    assert len(r) == 8                                  # only free entries are admitted
    assert len(sv.submit([i0], q1[20:21], p)) == 0
    out = [sv.wait(x, 10) for x in r]
    r2 = sv.submit(np.full(12, i0), q1[8:20], p)
    assert len(r2) == 8
    out += [sv.wait(x, 10) for x in r2]
    for j, o in enumerate(out):
        assert _same(o, _alone(ix1, q1[j], p))
    sv.close()


def test_server_admission_follows_free_memory(two_indexes):
    """Submits admit requests by the device memory that is free now: memory
    taken by someone else after the server was created lowers the admission
    cap below the ring, and giving it back raises it again."""
    import torch
    from falcon_b200.serving import FalconServer
    (ix1, q1), _ = two_indexes
    free0, _ = torch.cuda.mem_get_info()
    frac = 2000 * 600.0 / free0                         # a ring of about 2000 entries
    sv = FalconServer(ring_capacity=65536, max_k=10, ef_max=64, dim_max=128, idle_exit_us=2000,
                      memory_fraction=frac)
    i0 = sv.add_index(ix1)
    ring = sv.info().ring_entries
    assert 1000 < ring < 4000
    p = dict(k=10, ef=64)
    qs = np.ascontiguousarray(q1[np.arange(ring) % len(q1)])
    hog = torch.empty(int(free0 * 0.6), dtype=torch.uint8, device="cuda")
    time.sleep(0.1)                                     # the server re-reads free memory every few ms
    r = sv.submit(np.full(ring, i0), qs, p)
    assert 0 < len(r) < 0.6 * ring                      # ~40 % of the memory is free: ~40 % of the ring
    for x in r:
        sv.wait(x, 10)
    del hog
    torch.cuda.empty_cache()
    time.sleep(0.1)
    r2 = sv.submit(np.full(ring, i0), qs, p)
    assert len(r2) > 0.9 * ring
    for j, x in enumerate(r2):
        got = sv.wait(x, 10)
        if j < 8:
            assert _same(got, _alone(ix1, qs[j], p))
    sv.close()


def test_server_idle_exit_and_relaunch(two_indexes):
    from falcon_b200.serving import FalconServer
    (ix1, q1), _ = two_indexes
    sv = FalconServer(ring_capacity=64, max_k=10, ef_max=64, dim_max=128, idle_exit_us=200)
    i0 = sv.add_index(ix1)
    p = dict(k=10, ef=64, mg=2)
    a = sv.submit([i0], q1[:1], p)[0]
    ra = sv.wait(a, 10)
    time.sleep(0.05)                                    # the kernel leaves after 200 us idle
    b = sv.submit([i0], q1[1:2], p)[0]
    rb = sv.wait(b, 10)
    assert _same(ra, _alone(ix1, q1[0], p)) and _same(rb, _alone(ix1, q1[1], p))
    assert sv.info().kernel_launches >= 2
    sv.close()


def test_server_replay_poisson(two_indexes):
    from falcon_b200 import make_params
    from falcon_b200.serving import FalconServer, poisson_arrivals
    sv = FalconServer(ring_capacity=1024, max_k=50, ef_max=256, cand_queue_max=64, dim_max=384, idle_exit_us=3000)
    (ix1, _), (ix2, _) = two_indexes
    ids = [sv.add_index(ix1), sv.add_index(ix2)]
    reqs = _mixed_requests(two_indexes, 400, seed=2)
    dims = [128, 384]
    queries = np.zeros((len(reqs), 384), dtype=np.float32)
    for i, (w, q, p) in enumerate(reqs):
        queries[i, :dims[w]] = q
    # both indexes read only their own dimension from the padded rows
    arrival = poisson_arrivals(len(reqs), 20000.0, seed=3)
    lat, out_ids, out_d, hops, vis, el = sv.replay([ids[w] for w, _, _ in reqs], queries,
                                                   [make_params(**p) for _, _, p in reqs], arrival, 50)
    assert np.all(lat > 0) and el > 0
    for i, (w, q, p) in enumerate(reqs):
        got = (out_ids[i, :p["k"]], out_d[i, :p["k"]], int(hops[i]), int(vis[i]))
        assert _same(got, _alone(ix1 if w == 0 else ix2, q, p))
    sv.close()


def test_server_descends_upper_layers():
    """Requests to an index with HNSW upper layers start from the greedy
    descent of their own query (run on the copy stream at submit), like
    falcon_search without entry points: every served result equals the same
    request searched alone, FP32 and BF16 + rerank, in bursts and by replay."""
    from falcon_b200 import FalconIndex, make_params
    from falcon_b200.graph import build_graph, build_upper_layers
    from falcon_b200.serving import FalconServer, poisson_arrivals
    from falcon_b200.synthetic import unit_normal
    x = unit_normal(6000, 96, 41)
    q = unit_normal(96, 96, 42)
    g = build_graph(x, 64, device="cuda")
    upper = build_upper_layers(x, 32, seed=5, device="cuda")
    g.entry_point = upper.entry
    ix = FalconIndex(g, storage=("f32", "bf16"))
    ix.set_upper_layers(upper)
    sv = FalconServer(ring_capacity=512, max_k=10, ef_max=128, cand_queue_max=64, bloom_bits_max=17, dim_max=96,
                      idle_exit_us=3000)
    iid = sv.add_index(ix)
    params = [dict(k=10, ef=128, mc=2, mg=2, cand_queue_size=64, bloom_bits=17),
              dict(k=10, ef=96, cand_queue_size=32, bloom_bits=16, precision="bf16", rerank=True)]
    reqs = [(q[i], params[i % 2]) for i in range(len(q))]
    rids = []
    for s in range(0, len(reqs), 8):
        for qq, p in reqs[s:s + 8]:
            rids.append(sv.submit([iid], qq[None, :], p)[0])
    for (qq, p), rid in zip(reqs, rids):
        assert _same(sv.wait(rid, p["k"]), _alone(ix, qq, p)), p
    lat, ids, d, hops, vis, el = sv.replay(np.full(len(q), iid), q, [make_params(**p) for _, p in reqs],
                                           poisson_arrivals(len(q), 50000.0, seed=7), 10)
    for i, (qq, p) in enumerate(reqs):
        assert _same((ids[i], d[i], int(hops[i]), int(vis[i])), _alone(ix, qq, p)), (i, p)
    sv.close()
    ix.close()


def test_registered_index_cannot_be_freed_or_changed():
    """A server holds device pointers into its indexes: freeing a registered
    index or replacing its upper layers is refused until the server is freed."""
    from falcon_b200 import FalconIndex, _lib
    from falcon_b200.graph import build_upper_layers
    from falcon_b200.serving import FalconServer
    from falcon_b200.synthetic import unit_normal
    g, q = small_graph("unit", 2000, 64, 32, 8, seed=51)
    ix = FalconIndex(g, storage=("f32",))
    sv = FalconServer(ring_capacity=64, max_k=10, ef_max=64, dim_max=64, idle_exit_us=2000)
    iid = sv.add_index(ix)
    with pytest.raises(_lib.FalconError):
        ix.close()
    with pytest.raises(_lib.FalconError):
        ix.set_upper_layers(build_upper_layers(unit_normal(2000, 64, 51), 16, seed=1, device="cuda"))
    r = sv.submit([iid], q[:1], dict(k=10, ef=64))[0]
    assert _same(sv.wait(r, 10), _alone(ix, q[0], dict(k=10, ef=64)))
    sv.close()
    ix.close()
