"""Seeded synthetic stand-ins for the reference's datasets.

The reference measures on SIFT, Deep, SBERT and SPACEV (host.cpp:99-192),
which are not available here.  These generators reproduce their shapes and
value distributions:
  sift_like:  D=128, integers round(|N(0,40)|) clipped to [0, 255]
  deep_like:  D=96,  i.i.d. N(0,1) rows normalised to unit L2 norm
  sbert_like: D=384, i.i.d. N(0,1) rows normalised to unit L2 norm
Queries are drawn from the same distribution with a different seed.
"""
import numpy as np

WORKLOADS = {
    # name: (distribution, n_base, dim, n_queries, max_degree, defaults)
    "sift100k_hnsw_m16": ("sift", 100_000, 128, 1_000, 32, dict(k=10, ef=64, mc=1)),
    "deep1m_hnsw_m32": ("unit", 1_000_000, 96, 10_000, 64, dict(k=10, ef=64, mc=1)),
    "sift10m_nsg_r64": ("sift", 10_000_000, 128, 100_000, 64, dict(k=10, ef=64, mc=1)),
    "sbert1m_hnsw_m32": ("unit", 1_000_000, 384, 10_000, 64, dict(k=10, ef=64, mc=2)),
}


def sift_like(n, dim=128, seed=0, chunk=1 << 20):
    rng = np.random.default_rng(seed)
    out = np.empty((n, dim), dtype=np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        v = np.rint(np.abs(rng.normal(0.0, 40.0, size=(e - s, dim))))
        out[s:e] = np.clip(v, 0, 255)
    return out


def unit_normal(n, dim, seed=0, chunk=1 << 20):
    rng = np.random.default_rng(seed)
    out = np.empty((n, dim), dtype=np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        v = rng.standard_normal(size=(e - s, dim))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        out[s:e] = v
    return out


def _blocks(n, dim, seed, fill, threads=None, block=1 << 20):
    """Rows [b*block, (b+1)*block) come from their own generator seeded by
    (seed, b), so the result does not depend on how many threads fill it."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    out = np.empty((n, dim), dtype=np.float32)
    nb = (n + block - 1) // block

    def run(b):
        s, e = b * block, min(n, (b + 1) * block)
        fill(np.random.default_rng([seed, b]), out[s:e])

    with ThreadPoolExecutor(max_workers=threads or min(32, os.cpu_count() or 1)) as ex:
        list(ex.map(run, range(nb)))
    return out


def sift_like_blocks(n, dim=128, seed=0, threads=None):
    """sift_like's distribution from block-seeded generators filled in
    parallel (for bases of 10^7 rows); a different stream than sift_like."""
    def fill(rng, dst):
        v = np.rint(np.abs(rng.normal(0.0, 40.0, size=dst.shape)))
        np.clip(v, 0, 255, out=v)
        dst[...] = v
    return _blocks(n, dim, seed, fill, threads)


def unit_normal_blocks(n, dim, seed=0, threads=None):
    """unit_normal's distribution from block-seeded generators filled in
    parallel; a different stream than unit_normal."""
    def fill(rng, dst):
        v = rng.standard_normal(size=dst.shape)
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        dst[...] = v
    return _blocks(n, dim, seed, fill, threads)


def make(distribution, n, dim, seed):
    if distribution == "sift":
        return sift_like(n, dim, seed)
    if distribution == "unit":
        return unit_normal(n, dim, seed)
    raise ValueError(distribution)


def workload(name, n_base=None, n_queries=None, data_seed=0, query_seed=1):
    """Base vectors and queries of a named workload (optionally scaled down)."""
    dist, nb, dim, nq, md, defaults = WORKLOADS[name]
    nb = n_base or nb
    nq = n_queries or nq
    return make(dist, nb, dim, data_seed), make(dist, nq, dim, query_seed), md, dict(defaults)
