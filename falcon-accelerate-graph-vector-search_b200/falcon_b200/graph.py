"""Proximity-graph construction for the synthetic workloads.

The reference builds its graphs offline with hnswlib (HNSW) or the NSG tools
(vector_search_baselines/scripts_hnsw/construct_and_search_hnsw.py:124-153,
scripts_nsg/README_nsg.md) and the kernel only searches the base layer from
one entry point (host.cpp:711-713).  For workloads of 10^6+ points this module
builds an equivalent single-layer graph on the GPU:
  1. exact k-nearest-neighbour lists (chunked GEMM, top-k),
  2. hnswlib's neighbour-selection heuristic (hnswalg.h:328-369,
     getNeighborsByHeuristic2: keep a candidate only if it is closer to the
     node than to every neighbour already kept), capped at max_degree,
  3. reverse edges added and each row re-pruned with the same heuristic,
  4. the medoid (point nearest the mean) as the entry point, as NSG does.
It is data preparation, not the search path; torch is used for the bulk math.
"""
import numpy as np
import torch

from .formats import Graph


def _device(device):
    if device is not None:
        return torch.device(device)
    return torch.device("cuda" if torch.cuda.is_available() else "cpu")


def knn(vectors, k, device=None, chunk=None):
    """Exact k nearest neighbours of every row (self excluded): ids, sq. distances."""
    dev = _device(device)
    x = torch.from_numpy(np.ascontiguousarray(vectors, dtype=np.float32)).to(dev)
    n = x.shape[0]
    k = min(k, n - 1)
    norms = (x * x).sum(1)
    if chunk is None:
        chunk = max(256, min(8192, int(2e9 // max(1, n))))
    ids = torch.empty((n, k), dtype=torch.int64, device=dev)
    dst = torch.empty((n, k), dtype=torch.float32, device=dev)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for s in range(0, n, chunk):
            e = min(n, s + chunk)
            d = norms[s:e, None] - 2.0 * (x[s:e] @ x.T) + norms[None, :]
            d[torch.arange(e - s, device=dev), torch.arange(s, e, device=dev)] = float("inf")
            v, i = torch.topk(d, k, dim=1, largest=False, sorted=True)
            ids[s:e] = i
            dst[s:e] = v.clamp_min(0)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return ids, dst


def _heuristic_prune(x, node_ids, cand, cand_d, max_degree):
    """hnswlib getNeighborsByHeuristic2 over a batch.  cand sorted ascending by
    cand_d, -1 = empty.  Returns [B, max_degree] ids (-1 padded)."""
    b, kc = cand.shape
    valid = cand >= 0
    cv = x[cand.clamp_min(0)]                                  # [B, K, D]
    sq = (cv * cv).sum(-1)
    pair = sq[:, :, None] - 2.0 * torch.bmm(cv, cv.transpose(1, 2)) + sq[:, None, :]   # [B, K, K]
    kept = torch.zeros((b, kc), dtype=torch.bool, device=x.device)
    nkept = torch.zeros(b, dtype=torch.int64, device=x.device)
    for j in range(kc):
        # candidate j is rejected if some kept i has dist(i, j) < dist(j, node)
        closer = (pair[:, :j, j] < cand_d[:, j:j + 1]) & kept[:, :j]
        good = valid[:, j] & ~closer.any(1) & (nkept < max_degree)
        kept[:, j] = good
        nkept += good.long()
    out = torch.full((b, max_degree), -1, dtype=torch.int64, device=x.device)
    order = torch.argsort((~kept).to(torch.int8), dim=1, stable=True)[:, :max_degree]
    sel = torch.gather(cand, 1, order)
    selk = torch.gather(kept, 1, order)
    out[:, :sel.shape[1]] = torch.where(selk, sel, torch.full_like(sel, -1))
    return out


def _build_graph_cuda(xs, x, ids, max_degree):
    """Steps 2-3 with the library's neighbour-selection kernel
    (falcon_graph_prune, the same rule): forward prune of the kNN lists, then
    forward + reverse candidates pruned again."""
    from .nsg import prune, reverse_lists
    adj, _ = prune(x, ids.to(torch.int32), max_degree)
    rev = reverse_lists(adj, max_degree)
    adj, _ = prune(x, torch.cat([adj, rev], 1), max_degree)
    return adj


def build_graph(vectors, max_degree, knn_k=None, device=None, batch=2048, verbose=False):
    """Single-layer graph of max degree `max_degree` with medoid entry point.
    On a GPU the neighbour selection runs in the library's prune kernel; on
    the CPU in torch (same rule)."""
    dev = _device(device)
    xs = np.ascontiguousarray(vectors, dtype=np.float32)
    n = xs.shape[0]
    kk = min(knn_k or 2 * max_degree, n - 1)
    ids, dst = knn(xs, kk, device=dev)
    x = torch.from_numpy(xs).to(dev)
    if dev.type == "cuda" and 4 * kk * (((xs.shape[1] + 3) // 4) + 4) <= 200 * 1024:
        adj = _build_graph_cuda(xs, x, ids, max_degree)
        mean = x.mean(0, keepdim=True)
        entry = int(torch.argmin(((x - mean) ** 2).sum(1)).item())
        return Graph.from_adjacency(xs, adj.cpu().numpy(), entry)
    fwd = torch.empty((n, max_degree), dtype=torch.int64, device=dev)
    for s in range(0, n, batch):
        e = min(n, s + batch)
        fwd[s:e] = _heuristic_prune(x, None, ids[s:e], dst[s:e], max_degree)
    if verbose:
        print("forward edges done")
    # reverse edges: u -> v kept implies v gets candidate u
    src = torch.arange(n, device=dev)[:, None].expand(n, max_degree)
    m = fwd >= 0
    rv_dst, rv_src = fwd[m], src[m]
    order = torch.argsort(rv_dst, stable=True)
    rv_dst, rv_src = rv_dst[order], rv_src[order]
    counts = torch.bincount(rv_dst, minlength=n)
    starts = torch.cumsum(counts, 0) - counts
    rmax = max_degree   # cap the reverse candidates per node
    pos = torch.arange(rv_dst.numel(), device=dev) - starts[rv_dst]
    keep = pos < rmax
    rev = torch.full((n, rmax), -1, dtype=torch.int64, device=dev)
    rev[rv_dst[keep], pos[keep]] = rv_src[keep]
    out = torch.full((n, max_degree), -1, dtype=torch.int64, device=dev)
    for s in range(0, n, batch):
        e = min(n, s + batch)
        cand = torch.cat([fwd[s:e], rev[s:e]], dim=1)              # [B, 2*MD]
        # dedup: sort ids, mark repeats
        cs, _ = torch.sort(torch.where(cand >= 0, cand, torch.full_like(cand, n)), dim=1)
        dup = torch.zeros_like(cs, dtype=torch.bool)
        dup[:, 1:] = cs[:, 1:] == cs[:, :-1]
        cs = torch.where(dup | (cs >= n), torch.full_like(cs, -1), cs)
        cv = x[cs.clamp_min(0)]
        d = ((cv - x[s:e, None, :]) ** 2).sum(-1)
        d = torch.where(cs >= 0, d, torch.full_like(d, float("inf")))
        dsort, o = torch.sort(d, dim=1, stable=True)
        csort = torch.gather(cs, 1, o)
        out[s:e] = _heuristic_prune(x, None, csort, dsort, max_degree)
    mean = x.mean(0, keepdim=True)
    entry = int(torch.argmin(((x - mean) ** 2).sum(1)).item())
    adj = out.to(torch.int32).cpu().numpy()
    return Graph.from_adjacency(xs, adj, entry)


def build_upper_layers(vectors, M, seed=0, device=None):
    """HNSW upper layers for a base graph over `vectors`: node levels drawn as
    hnswlib draws them (floor(-ln U * mult), mult = 1/ln M; hnswalg.h:148-153,
    here from a seeded numpy generator), and on every level l >= 1 a graph of
    max degree M over the nodes with level >= l, built like the base layer
    (k nearest neighbours, hnswlib's heuristic, reverse edges).  The entry is
    the medoid of the top level.  Returns formats.UpperLayers."""
    from .formats import UpperLayers
    xs = np.ascontiguousarray(vectors, dtype=np.float32)
    n = xs.shape[0]
    rng = np.random.default_rng(seed)
    mult = 1.0 / np.log(float(M))
    u = rng.random(n)
    levels = np.floor(-np.log(np.maximum(u, 1e-300)) * mult).astype(np.int32)
    max_level = int(levels.max())
    if max_level < 1:   # make sure there is one upper level with one node
        levels[int(rng.integers(0, n))] = 1
        max_level = 1
    lists = [[] for _ in range(n)]
    entry = -1
    for lvl in range(1, max_level + 1):
        nodes = np.nonzero(levels >= lvl)[0]
        if nodes.size == 1:
            lists[int(nodes[0])].append(np.zeros(0, dtype=np.int32))
            entry = int(nodes[0])
            continue
        sub = build_graph(xs[nodes], min(M, nodes.size - 1), device=device)
        adj = sub.adjacency()
        for j, v in enumerate(nodes):
            row = adj[j]
            lists[int(v)].append(nodes[row[row >= 0]].astype(np.int32))
        entry = int(nodes[sub.entry_point])
    return UpperLayers.from_lists(M, entry, lists)
