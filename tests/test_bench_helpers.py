"""CPU: the bench's accounting helpers (algorithmic bytes per query, distance
error against FP64) on hand-checked inputs."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def test_algorithmic_bytes():
    import bench
    hops = np.array([10, 20])
    vis = np.array([100, 300])
    ks = np.array([1, 100])
    D, R = 128, 64
    # per query: visited * D * 4 + hops * (4 + 4 * degree) + D * 4 (query) + k * 8 (results)
    per = lambda h, v, k: v * D * 4 + h * (4 + 4 * R) + D * 4 + k * 8
    assert bench.algorithmic_bytes(hops, vis, D, R, ks) == per(10, 100, 1) + per(20, 300, 100)
    # BF16 gathers half the bytes; the rerank reads ef FP32 vectors; D=96 pads to 96
    efs = np.array([64, 128])
    b16 = bench.algorithmic_bytes(hops, vis, 96, R, ks, efs, elem_bytes=2, rerank=True)
    assert b16 == sum(v * 96 * 2 + h * (4 + 4 * R) + ef * 96 * 4 + 96 * 4 + k * 8
                      for h, v, k, ef in ((10, 100, 1, 64), (20, 300, 100, 128)))
    # FP8: one byte per padded dimension plus a 4-byte scale per vector; D=100 pads to 112
    f8 = bench.algorithmic_bytes(hops, vis, 100, R, ks, elem_bytes=1, scale_bytes=4)
    assert f8 == sum(v * (112 + 4) + h * (4 + 4 * R) + 100 * 4 + k * 8 for h, v, k in ((10, 100, 1), (20, 300, 100)))


def test_mixed_recall_groups():
    import bench
    gt = np.tile(np.arange(100), (4, 1))
    ids = np.full((4, 100), -1)
    ids[0, :10] = np.arange(10)          # k=10, all found
    ids[1, :1] = [5]                     # k=1, wrong
    ids[2, :100] = np.arange(100)        # k=100, all found
    ids[3, :10] = np.arange(5, 15)       # k=10, half found
    r = bench.mixed_recall(ids, gt, np.array([10, 1, 100, 10]))
    assert r["recall@1_k=1"] == 0.0
    assert r["recall@100_k=100"] == 1.0
    assert abs(r["recall@10_k>=10"] - (10 + 10 + 5) / 30.0) < 1e-12


def test_sift10m_params_seeded():
    import bench
    e1, k1, m1 = bench.sift10m_params(1000)
    e2, k2, m2 = bench.sift10m_params(1000)
    assert np.array_equal(e1, e2) and np.array_equal(k1, k2) and np.array_equal(m1, m2)
    assert set(np.unique(k1)) == {1, 10, 100} and set(np.unique(m1)) == {1, 2, 4}
    assert (e1 >= k1).all() and set(np.unique(e1)) <= {32, 64, 100, 128, 256}


def test_distance_error_f64():
    import bench
    rng = np.random.default_rng(1)
    x = rng.standard_normal((50, 8)).astype(np.float32)
    q = rng.standard_normal((3, 8)).astype(np.float32)
    ids = np.array([[0, 5, -1], [7, 8, 9], [1, -1, -1]])
    exact = np.zeros(ids.shape)
    for i in range(3):
        for j in range(3):
            if ids[i, j] >= 0:
                exact[i, j] = ((x[ids[i, j]].astype(np.float64) - q[i]) ** 2).sum()
    e = bench.distance_error_f64(x, q, ids, exact)
    assert e["max_rel"] == 0.0 and e["mean_rel"] == 0.0
    e = bench.distance_error_f64(x, q, ids, exact * (1 + 1e-3))
    assert abs(e["max_rel"] - 1e-3) < 1e-9


def test_traffic_record_follows_the_kernel_source(tmp_path, monkeypatch):
    """roofline.traffic comes from profiles/traffic.json only while the
    recorded capture was taken on the current kernel source; the committed
    record covers both workloads the bench applies it to."""
    import hashlib
    import json
    import bench
    src = os.path.join(bench.REPO, "falcon-accelerate-graph-vector-search_b200", "csrc", "falcon_kernels.cu")
    h = hashlib.sha256(open(src, "rb").read()).hexdigest()[:16]
    rec = json.load(open(os.path.join(bench.REPO, "profiles", "traffic.json")))
    for key in ("sift10m_mixed", "deep1m_f32_throughput_point"):
        assert rec[key]["kernel_source_sha16"] == h
        roof = {}
        bench.traffic_from_profile(roof, key, 1000.0)
        assert abs(roof["traffic"] - rec[key]["ratio"] * 1000.0) < 1e-9
    # a record of another source is not applied
    fake = tmp_path / "repo"
    (fake / "profiles").mkdir(parents=True)
    (fake / "falcon-accelerate-graph-vector-search_b200" / "csrc").mkdir(parents=True)
    (fake / "falcon-accelerate-graph-vector-search_b200" / "csrc" / "falcon_kernels.cu").write_text("changed")
    (fake / "profiles" / "traffic.json").write_text(json.dumps(rec))
    monkeypatch.setattr(bench, "REPO", str(fake))
    roof = {}
    bench.traffic_from_profile(roof, "sift10m_mixed", 1000.0)
    assert "traffic" not in roof and "no ncu capture" in roof["traffic_note"]
