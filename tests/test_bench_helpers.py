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
    # per query: visited * D * 4 + hops * (4 + 4 * degree) + D * 4 (query) + k * 8 (results)
    per = lambda h, v: v * bench.DIM * 4 + h * (4 + 4 * bench.MAX_DEGREE) + bench.DIM * 4 + bench.K * 8
    assert bench.algorithmic_bytes(hops, vis, 64) == per(10, 100) + per(20, 300)
    # BF16 gathers half the bytes; the rerank reads ef FP32 vectors
    b16 = bench.algorithmic_bytes(hops, vis, 64, elem_bytes=2, rerank=True)
    assert b16 == sum(v * bench.DIM * 2 + h * (4 + 4 * bench.MAX_DEGREE) + 64 * bench.DIM * 4 + bench.DIM * 4
                      + bench.K * 8 for h, v in ((10, 100), (20, 300)))


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
