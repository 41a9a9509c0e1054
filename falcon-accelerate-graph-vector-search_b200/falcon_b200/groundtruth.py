"""FP64 ground truth and recall scoring on the host.

Recall@k follows the reference host (host.cpp:1010-1068): for each of the k
ground-truth ids, count it if it appears among the first k returned ids.
"""
import numpy as np


def brute_force_f64(base, queries, k, chunk=256):
    """Exact top-k by FP64 squared L2 over all base vectors (host, numpy)."""
    b = np.asarray(base, dtype=np.float64)
    bn = (b * b).sum(1)
    out_i = np.empty((len(queries), k), dtype=np.int64)
    out_d = np.empty((len(queries), k), dtype=np.float64)
    for s in range(0, len(queries), chunk):
        q = np.asarray(queries[s:s + chunk], dtype=np.float64)
        d = (q * q).sum(1)[:, None] - 2.0 * (q @ b.T) + bn[None, :]
        part = np.argpartition(d, k - 1, axis=1)[:, :k]
        dp = np.take_along_axis(d, part, 1)
        o = np.argsort(dp, axis=1, kind="stable")
        out_i[s:s + chunk] = np.take_along_axis(part, o, 1)
        out_d[s:s + chunk] = np.take_along_axis(dp, o, 1)
    # exact FP64 distances of the winners (not the expanded-norm form)
    diff = b[out_i] - np.asarray(queries, dtype=np.float64)[:, None, :]
    out_d = (diff * diff).sum(-1)
    o = np.argsort(out_d, axis=1, kind="stable")
    return np.take_along_axis(out_i, o, 1), np.take_along_axis(out_d, o, 1)


def shortlist_f64(base, queries, k, shortlist=64, device=None):
    """FP64 ground truth for large bases: an FP32 GPU shortlist of `shortlist`
    candidates per query, then exact FP64 distances computed on the host and
    re-sorted.  Equal to brute_force_f64 whenever the true top-k lies in the
    FP32 top-`shortlist` (FP32 error is ~1e-7 relative)."""
    import torch
    dev = torch.device(device or ("cuda" if torch.cuda.is_available() else "cpu"))
    x = torch.from_numpy(np.ascontiguousarray(base, dtype=np.float32)).to(dev)
    xn = (x * x).sum(1)
    cand = np.empty((len(queries), shortlist), dtype=np.int64)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for s in range(0, len(queries), 1024):
            q = torch.from_numpy(np.ascontiguousarray(queries[s:s + 1024], dtype=np.float32)).to(dev)
            d = (q * q).sum(1)[:, None] - 2.0 * (q @ x.T) + xn[None, :]
            cand[s:s + len(q)] = torch.topk(d, shortlist, dim=1, largest=False).indices.cpu().numpy()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    b = np.asarray(base)
    q64 = np.asarray(queries, dtype=np.float64)
    d64 = np.empty(cand.shape, dtype=np.float64)
    for s in range(0, len(queries), 4096):
        diff = b[cand[s:s + 4096]].astype(np.float64) - q64[s:s + 4096, None, :]
        d64[s:s + 4096] = (diff * diff).sum(-1)
    o = np.argsort(d64, axis=1, kind="stable")[:, :k]
    return np.take_along_axis(cand, o, 1), np.take_along_axis(d64, o, 1)


def shortlist_f64_tiled(base, queries, k, shortlist=64, base_device=None, q_chunk=2048, b_chunk=1 << 20,
                        device=None):
    """shortlist_f64 for bases of 10^7 rows: the FP32 shortlist is formed
    tile by tile (q_chunk queries x b_chunk base rows per GEMM, running top
    `shortlist` merged across tiles), then rescored in FP64 on the host.
    base_device: the base already on the GPU (optional)."""
    import torch
    dev = torch.device(device or "cuda")
    x = base_device if base_device is not None else torch.from_numpy(np.ascontiguousarray(base, dtype=np.float32)).to(dev)
    xn = (x * x).sum(1)
    n = x.shape[0]
    cand = np.empty((len(queries), shortlist), dtype=np.int64)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for s in range(0, len(queries), q_chunk):
            q = torch.from_numpy(np.ascontiguousarray(queries[s:s + q_chunk], dtype=np.float32)).to(dev)
            qn = (q * q).sum(1)
            bv = bi = None
            for b in range(0, n, b_chunk):
                d = qn[:, None] - 2.0 * (q @ x[b:b + b_chunk].T) + xn[None, b:b + b_chunk]
                v, i = torch.topk(d, min(shortlist, d.shape[1]), dim=1, largest=False)
                i = i + b
                if bv is not None:
                    v, i = torch.cat([bv, v], 1), torch.cat([bi, i], 1)
                    o = torch.topk(v, min(shortlist, v.shape[1]), dim=1, largest=False).indices
                    v, i = torch.gather(v, 1, o), torch.gather(i, 1, o)
                bv, bi = v, i
            cand[s:s + len(q)] = bi.cpu().numpy()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    b = np.asarray(base)
    q64 = np.asarray(queries, dtype=np.float64)
    d64 = np.empty(cand.shape, dtype=np.float64)
    for s in range(0, len(queries), 4096):
        diff = b[cand[s:s + 4096]].astype(np.float64) - q64[s:s + 4096, None, :]
        d64[s:s + 4096] = (diff * diff).sum(-1)
    o = np.argsort(d64, axis=1, kind="stable")[:, :k]
    return np.take_along_axis(cand, o, 1), np.take_along_axis(d64, o, 1)


def recall_at_k(found_ids, gt_ids, k=10):
    """Fraction of the k ground-truth ids found among the first k results."""
    f = np.asarray(found_ids)[:, :k]
    g = np.asarray(gt_ids)[:, :k]
    hits = 0
    for i in range(len(g)):
        hits += len(np.intersect1d(f[i], g[i], assume_unique=False))
    return hits / float(g.size)


def recall_at_1(found_ids, gt_ids):
    return float(np.mean(np.asarray(found_ids)[:, 0] == np.asarray(gt_ids)[:, 0]))
