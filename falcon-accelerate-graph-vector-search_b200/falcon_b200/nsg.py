"""NSG-style graph construction on the GPU for bases of 10^7 vectors.

The reference builds its NSG graphs offline with the NSG tool
(vector_search_baselines/scripts_nsg/README_nsg.md: an efanna kNN graph, then
NSG's candidate search, occlusion prune to R and reverse-edge insertion,
converted by scripts_nsg/nsg_to_FPGA.py:56-137) and searches them from a
fixed medoid entry point.  The tool is not vendored, so this module builds an
equivalent single-layer graph of max degree R on one GPU:

  1. approximate k nearest neighbours from an inverted file: k-means
     centroids (seeded), every point assigned to its nearest centroid, and
     each cluster's points compared exactly against the points of its
     `n_probe` nearest clusters (GEMM + top-k per cluster);
  2. occlusion prune of every node's candidates to R neighbours
     (falcon_graph_prune: hnswlib's / NSG's rule, alpha = 1);
  3. reverse edges: every kept edge u -> v offers u to v, and each node's
     forward and reverse candidates are pruned again;
  4. NSG's search step, repeated per pass: every node is searched on the
     graph so far (this library's own traversal kernel, from the medoid) and
     its ef best results join its candidates for another prune + reverse
     round; a pass may prune with alpha > 1 (keep a candidate unless
     alpha * d(kept, c) < d(c, node)), which keeps the longer edges that
     high-dimensional data needs to stay navigable (DiskANN's second pass);
  5. the medoid (the point nearest the mean) as the entry point, and a
     breadth-first search from it; nodes it does not reach are attached to the
     first reached node of their candidate list, as NSG attaches unreached
     nodes to its spanning tree.

Nodes are pruned grouped by cluster so that the candidate vectors of the
thread blocks in flight stay in L2.  It is data preparation, not the search
path: torch does the bulk GEMMs and sorts, the prune is this library's kernel.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib
from .formats import Graph


def _log(verbose, *a):
    if verbose:
        import sys
        print(*a, file=sys.stderr, flush=True)


def _sqdist_block(xa, na, xb, nb):
    """[a, b] squared distances from norms and one GEMM."""
    return (na[:, None] + nb[None, :]) - 2.0 * (xa @ xb.T)


def kmeans(x, xn, n_clusters, iters=6, sample=None, seed=1, chunk=65536):
    """Lloyd's k-means on a seeded sample of the rows of x (device tensor);
    returns the centroids [C, d]."""
    n = x.shape[0]
    g = torch.Generator(device="cpu")
    g.manual_seed(int(seed))
    m = min(n, sample or 64 * n_clusters)
    sel = torch.randperm(n, generator=g)[:m].to(x.device)
    xs, xsn = x[sel], xn[sel]
    cent = xs[torch.randperm(m, generator=g)[:n_clusters].to(x.device)].clone()
    for _ in range(iters):
        cn = (cent * cent).sum(1)
        lab = torch.empty(m, dtype=torch.int64, device=x.device)
        for s in range(0, m, chunk):
            lab[s:s + chunk] = torch.argmin(_sqdist_block(xs[s:s + chunk], xsn[s:s + chunk], cent, cn), dim=1)
        cnt = torch.bincount(lab, minlength=n_clusters).to(x.dtype)
        acc = torch.zeros_like(cent).index_add_(0, lab, xs)
        nz = cnt > 0
        cent[nz] = acc[nz] / cnt[nz, None]
    return cent


def assign(x, xn, cent, chunk=65536):
    cn = (cent * cent).sum(1)
    lab = torch.empty(x.shape[0], dtype=torch.int64, device=x.device)
    for s in range(0, x.shape[0], chunk):
        lab[s:s + chunk] = torch.argmin(_sqdist_block(x[s:s + chunk], xn[s:s + chunk], cent, cn), dim=1)
    return lab


def ivf_knn(x, k, n_clusters, n_probe, seed=1, xn=None, iters=6, row_chunk=4096, verbose=False):
    """Approximate k nearest neighbours (self excluded) of every row of the
    device tensor x: exact distances to the points of each cluster's n_probe
    nearest clusters.  Returns (ids [n, k] int32, cluster order [n] int64)."""
    t0 = time.time()
    n = x.shape[0]
    if xn is None:
        xn = (x * x).sum(1)
    cent = kmeans(x, xn, n_clusters, iters=iters, seed=seed)
    lab = assign(x, xn, cent)
    order = torch.argsort(lab, stable=True)
    cnt = torch.bincount(lab, minlength=n_clusters)
    off = np.zeros(n_clusters + 1, dtype=np.int64)
    off[1:] = np.cumsum(cnt.cpu().numpy())
    cn = (cent * cent).sum(1)
    probe = torch.topk(_sqdist_block(cent, cn, cent, cn), min(n_probe, n_clusters), dim=1,
                       largest=False).indices.cpu().numpy()
    _log(verbose, "ivf: k-means + assignment %.1fs (clusters %d, largest %d)" % (time.time() - t0, n_clusters,
                                                                                int(cnt.max())))
    t0 = time.time()
    out = torch.full((n, k), -1, dtype=torch.int32, device=x.device)
    for c in range(n_clusters):
        a, b = int(off[c]), int(off[c + 1])
        if a == b:
            continue
        members = order[a:b]
        cand = torch.cat([order[int(off[p]):int(off[p + 1])] for p in probe[c]])
        xc, xcn = x[cand], xn[cand]
        kk = min(k, cand.numel() - 1)
        if kk <= 0:
            continue
        for s in range(0, b - a, row_chunk):
            m = members[s:s + row_chunk]
            d = _sqdist_block(x[m], xn[m], xc, xcn)
            d.masked_fill_(m[:, None] == cand[None, :], float("inf"))
            idx = torch.topk(d, kk, dim=1, largest=False, sorted=False).indices
            out[m, :kk] = cand[idx].to(torch.int32)
    _log(verbose, "ivf: per-cluster kNN %.1fs" % (time.time() - t0))
    return out, order


def prune(x, cand, max_degree, alpha=1.0, order=None, stream=None):
    """falcon_graph_prune over every node: cand [n, K] int32 device tensor ->
    [n, max_degree] int32 (nearest first, -1 padded), counts [n]."""
    lib = _lib.load()
    n, K = cand.shape
    cand = cand.contiguous()
    out = torch.empty((n, max_degree), dtype=torch.int32, device=x.device)
    cnt = torch.empty(n, dtype=torch.int32, device=x.device)
    nodes = None if order is None else order.to(torch.int32).contiguous()
    s = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
    _lib.check(lib.falcon_graph_prune(x.data_ptr(), n, x.shape[1], x.stride(0), cand.data_ptr(), cand.stride(0), K,
                                      nodes.data_ptr() if nodes is not None else None, n, ctypes.c_float(alpha),
                                      max_degree, out.data_ptr(), out.stride(0), cnt.data_ptr(),
                                      x.device.index or 0, ctypes.c_void_p(s)))
    return out, cnt


def reverse_lists(adj, cap):
    """[n, cap] int32: for every node v up to `cap` sources u of kept edges
    u -> v (in ascending u), -1 padded."""
    n, r = adj.shape
    dev = adj.device
    m = adj >= 0
    dst = adj[m].to(torch.int64)
    src = torch.arange(n, device=dev, dtype=torch.int32)[:, None].expand(n, r)[m]
    dst, perm = torch.sort(dst, stable=True)
    src = src[perm]
    del perm
    counts = torch.bincount(dst, minlength=n)
    starts = torch.cumsum(counts, 0) - counts
    pos = torch.arange(dst.numel(), device=dev) - starts[dst]
    keep = pos < cap
    rev = torch.full((n, cap), -1, dtype=torch.int32, device=dev)
    rev[dst[keep], pos[keep]] = src[keep]
    return rev


def reachable(adj, entry):
    """Boolean [n]: nodes a breadth-first search from `entry` reaches."""
    n = adj.shape[0]
    seen = torch.zeros(n, dtype=torch.bool, device=adj.device)
    seen[entry] = True
    frontier = torch.tensor([entry], dtype=torch.int64, device=adj.device)
    while frontier.numel():
        nb = adj[frontier].reshape(-1)
        nb = nb[nb >= 0].to(torch.int64)
        nb = torch.unique(nb[~seen[nb]])
        seen[nb] = True
        frontier = nb
    return seen


def attach_unreached(adj, cnt, seen, cand, entry, rounds=16):
    """Give every node the breadth-first search misses an in-edge: from the
    first reached node of its candidate list that has a free slot, else from
    any reached node with a free slot, else over the farthest edge of its
    first reached candidate; repeat until all are reached.  adj/cnt are
    updated in place.  Returns (edges added, reachability)."""
    added = 0
    R = adj.shape[1]
    dev = adj.device
    for _ in range(rounds):
        un = torch.nonzero(~seen).flatten()
        if un.numel() == 0:
            break
        c = cand[un].to(torch.int64)
        cc = c.clamp_min(0)
        reached = (c >= 0) & seen[cc]
        free = reached & (cnt[cc] < R)
        rows = torch.arange(un.numel(), device=dev)
        w = torch.where(free.any(1), cc[rows, torch.argmax(free.to(torch.int8), 1)], torch.full_like(un, -1))
        pool = torch.nonzero(seen & (cnt < R)).flatten()
        miss = w < 0
        if miss.any() and pool.numel():
            w[miss] = pool[torch.arange(int(miss.sum()), device=dev) % pool.numel()]
        # the rest replace the farthest edge of their first reached candidate (or the entry's)
        miss = w < 0
        if miss.any():
            fr = torch.where(reached.any(1), cc[rows, torch.argmax(reached.to(torch.int8), 1)],
                             torch.full_like(un, int(entry)))
            adj[fr[miss], R - 1] = un[miss].to(adj.dtype)
            added += int(miss.sum())
        ok = w >= 0
        wv, uv = w[ok], un[ok]
        if wv.numel():
            wv, o = torch.sort(wv, stable=True)
            uv = uv[o]
            first = torch.ones_like(wv, dtype=torch.bool)
            first[1:] = wv[1:] != wv[:-1]
            start = torch.cummax(torch.where(first, torch.arange(wv.numel(), device=dev), torch.zeros_like(wv)), 0).values
            slot = cnt[wv].to(torch.int64) + (torch.arange(wv.numel(), device=dev) - start)
            fit = slot < R
            adj[wv[fit], slot[fit]] = uv[fit].to(adj.dtype)
            cnt.index_add_(0, wv[fit], torch.ones_like(wv[fit], dtype=cnt.dtype))
            added += int(fit.sum())
        seen = reachable(adj, entry)
    return added, seen


def medoid(x, chunk=1 << 20):
    mean = x.mean(0, keepdim=True)
    best_d, best_i = float("inf"), 0
    for s in range(0, x.shape[0], chunk):
        d = ((x[s:s + chunk] - mean) ** 2).sum(1)
        v, i = torch.min(d, 0)
        if float(v) < best_d:
            best_d, best_i = float(v), s + int(i)
    return best_i


def knn_recall(x, xn, approx, sample=1000, seed=1):
    """Recall of the approximate lists against exact neighbours on a sample."""
    n, k = approx.shape
    g = torch.Generator(device="cpu")
    g.manual_seed(int(seed) + 7)
    sel = torch.randperm(n, generator=g)[:min(sample, n)].to(x.device)
    best = None
    for s in range(0, n, 1 << 21):
        d = _sqdist_block(x[sel], xn[sel], x[s:s + (1 << 21)], xn[s:s + (1 << 21)])
        ids = torch.arange(s, min(n, s + (1 << 21)), device=x.device)
        d.masked_fill_(sel[:, None] == ids[None, :], float("inf"))
        v, i = torch.topk(d, k, dim=1, largest=False)
        i = ids[i]
        if best is None:
            best = (v, i)
        else:
            vv, ii = torch.cat([best[0], v], 1), torch.cat([best[1], i], 1)
            o = torch.topk(vv, k, dim=1, largest=False).indices
            best = (torch.gather(vv, 1, o), torch.gather(ii, 1, o))
    a = approx[sel].to(torch.int64)
    hit = (a[:, :, None] == best[1][:, None, :]).any(1).float().mean()
    return float(hit)


def build_nsg(vectors, max_degree=64, seed=1, knn_k=64, n_clusters=None, n_probe=24, alpha=1.0, search_passes=(),
              device=None, verbose=False, vectors_device=None, stats=None):
    """NSG-style single-layer graph of max degree `max_degree` over `vectors`
    (host [n, d] float32), medoid entry point.  search_passes: (ef, alpha)
    pairs, each one round of NSG's search step (every node searched on the
    graph so far at that ef; its results join its candidates) pruned with
    that alpha.  vectors_device: the same rows already on the GPU (optional).
    Returns a formats.Graph; `stats` (dict) receives timings and graph
    figures."""
    st = stats if stats is not None else {}
    dev = torch.device(device or "cuda")
    t_all = time.time()
    xs = np.ascontiguousarray(vectors, dtype=np.float32)
    n, dim = xs.shape
    x = vectors_device if vectors_device is not None else torch.from_numpy(xs).to(dev)
    xn = (x * x).sum(1)
    if n_clusters is None:
        n_clusters = max(1, min(16384, n // 512))
    prev_tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True   # candidate generation only; the prune recomputes in FP32
    try:
        t = time.time()
        knn, order = ivf_knn(x, min(knn_k, n - 1), n_clusters, n_probe, seed=seed, xn=xn, verbose=verbose)
        st["knn_s"] = time.time() - t
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev_tf32
    if n <= 2_000_000 or verbose:
        st["knn_recall"] = knn_recall(x, xn, knn)
        _log(verbose, "ivf kNN recall@%d %.3f" % (knn.shape[1], st["knn_recall"]))
    t = time.time()
    adj, cnt = prune(x, knn, max_degree, alpha, order)
    rev = reverse_lists(adj, max_degree)
    adj, cnt = prune(x, torch.cat([adj, rev], 1), max_degree, alpha, order)
    del rev
    torch.cuda.synchronize(dev)
    st["prune_s"] = time.time() - t
    entry = medoid(x)
    st["mean_degree_ivf"] = float(cnt.float().mean())
    for i, (ef_s, alpha_s) in enumerate(search_passes):
        t = time.time()
        cand = _search_candidates(xs, x, adj, entry, int(ef_s), dev)
        adj2, _ = prune(x, torch.cat([cand, adj], 1), max_degree, float(alpha_s), order)
        del cand
        rev = reverse_lists(adj2, max_degree)
        adj, cnt = prune(x, torch.cat([adj2, rev], 1), max_degree, float(alpha_s), order)
        del adj2, rev
        torch.cuda.synchronize(dev)
        st["search_pass_%d_s" % i] = time.time() - t
        st["mean_degree_pass_%d" % i] = float(cnt.float().mean())
        _log(verbose, "search pass %d (ef %d, alpha %.2f): %.1fs, mean degree %.1f" % (
            i, ef_s, alpha_s, time.time() - t, st["mean_degree_pass_%d" % i]))
    t = time.time()
    seen = reachable(adj, entry)
    st["unreached_before"] = int((~seen).sum())
    st["edges_added"], seen = attach_unreached(adj, cnt, seen, knn, entry)
    st["unreached_after"] = int((~seen).sum())
    st["connect_s"] = time.time() - t
    st["mean_degree"] = float(cnt.float().mean())
    adj_h = adj.cpu().numpy()
    del adj, knn, cnt, order
    if vectors_device is None:
        del x
    torch.cuda.empty_cache()
    st["entry"] = int(entry)
    st["build_s"] = time.time() - t_all
    st.update(dict(n_clusters=n_clusters, n_probe=n_probe, knn_k=knn_k, alpha=alpha,
                   search_passes=[list(p) for p in search_passes], seed=seed))
    _log(verbose, "nsg build %.1fs: %s" % (st["build_s"], {k: (round(v, 3) if isinstance(v, float) else v)
                                                          for k, v in st.items()}))
    return Graph.from_adjacency(xs, adj_h, entry)


def _search_candidates(xs, x, adj, entry, ef, dev, chunk=1 << 21):
    """NSG's candidate acquisition: every node searched on the current graph
    (FP32 inter-query traversal from the medoid, cand queue 64, 2^17-bit
    filter in shared memory); its ef results (itself excluded by the prune)
    as candidates."""
    from .index import FalconIndex
    g = Graph.from_adjacency(xs, adj.cpu().numpy(), entry)
    ix = FalconIndex(g, device=dev.index or 0)
    n = xs.shape[0]
    out = torch.empty((n, ef), dtype=torch.int32, device=dev)
    for s in range(0, n, chunk):
        r = ix.search(x[s:s + chunk], k=ef, ef=ef, mc=1, mg=1, cand_queue_size=64, bloom_bits=17)
        out[s:s + chunk] = r.ids
    torch.cuda.synchronize(dev)
    ix.close()
    return out
