"""Host-side mirror of the reference's search interface over the C ABI.

The reference host (FPGA_multi_DDR/FPGA_inter_query_v1.3_longer_FIFO_alt_PR/
src/host.cpp:34-96) takes mc (max_cand_per_group), mg
(max_group_num_in_pipe), ef, the graph and its max degree, then launches the
kernel once over all queries and reads back ids, distances and per-query
debug counters (hops, visited).  FalconIndex.search keeps those names and
outputs; everything runs in libfalcon_b200.so.
"""
import ctypes

import numpy as np

from . import _lib
from .formats import Graph

_PREC = {"f32": _lib.PREC_F32, "bf16": _lib.PREC_BF16, "fp8": _lib.PREC_FP8}
_MODE = {"inter": _lib.MODE_INTER, "intra": _lib.MODE_INTRA}
_STORE = {"f32": _lib.STORE_F32, "bf16": _lib.STORE_BF16, "fp8": _lib.STORE_FP8}


def storage_mask(storage):
    if isinstance(storage, int):
        return storage
    m = 0
    for s in storage:
        m |= _STORE[s]
    return m


def make_params(k=10, ef=64, mc=1, mg=1, cand_queue_size=32, bloom_bits=16, hash_seed=1, mode="inter",
                channels=4, precision="f32", rerank=False, max_hops=0):
    p = _lib.SearchParams()
    p.k, p.ef, p.mc, p.mg = int(k), int(ef), int(mc), int(mg)
    p.cand_queue_size, p.bloom_bits, p.hash_seed = int(cand_queue_size), int(bloom_bits), int(hash_seed)
    p.mode = _MODE[mode] if isinstance(mode, str) else int(mode)
    p.channels = int(channels)
    p.precision = _PREC[precision] if isinstance(precision, str) else int(precision)
    p.rerank = 1 if rerank else 0
    p.max_hops = int(max_hops)
    return p


def params_array(per_query):
    """A ctypes array of SearchParams from SearchParams or keyword dicts (one
    per query); build it once and pass it to search(per_query=...) to keep the
    conversion out of repeated calls."""
    arr = (_lib.SearchParams * len(per_query))()
    for i, p in enumerate(per_query):
        arr[i] = p if isinstance(p, _lib.SearchParams) else make_params(**p)
    return arr


def max_k(arr):
    ks = np.frombuffer(arr, dtype=np.int32).reshape(len(arr), ctypes.sizeof(_lib.SearchParams) // 4)[:, 0]
    return int(ks.max())


class SearchResult:
    def __init__(self, ids, dists, hops, visited, status):
        self.ids, self.dists, self.hops, self.visited, self.status = ids, dists, hops, visited, status

    def __iter__(self):
        return iter((self.ids, self.dists, self.hops, self.visited))


class Trace:
    """Per-query traversal trace: cand_d/cand_n [nq, cand_capacity] (distance
    of each expanded candidate, 1e20 for the entry, and the distances computed
    for its row), d/ids [nq, capacity] (each computed distance and its id, in
    traversal order), counts [nq, 3] (popped incl. entry, expanded, computed)."""

    def __init__(self, cand_d, cand_n, d, ids, counts):
        self.cand_d, self.cand_n, self.d, self.ids, self.counts = cand_d, cand_n, d, ids, counts

    def query(self, i):
        """(cand_d, cand_n, d, ids) of query i, cut to what was written."""
        ne = min(int(self.counts[i, 1]), self.cand_d.shape[1])
        nd = min(int(self.counts[i, 2]), self.d.shape[1])
        return self.cand_d[i, :ne], self.cand_n[i, :ne], self.d[i, :nd], self.ids[i, :nd]

    def reference_streams(self):
        """The reference trace kernel's flat outputs (debug_out_per_query_*,
        eval_trace_FPGA_inter_query_v1.3 DRAM_utils.hpp:389-404): per query -1,
        the entries, then -2; returns (cand_dists, cand_num_neighbors, dists, ids)."""
        cds, cns, ds, ids = [], [], [], []
        for i in range(self.counts.shape[0]):
            c_d, c_n, d, di = self.query(i)
            cds += [-1.0] + c_d.tolist() + [-2.0]
            cns += [-1] + c_n.tolist() + [-2]
            ds += [-1.0] + d.tolist() + [-2.0]
            ids += [-1] + di.tolist() + [-2]
        return (np.array(cds, dtype=np.float32), np.array(cns, dtype=np.int32), np.array(ds, dtype=np.float32),
                np.array(ids, dtype=np.int32))


class FalconIndex:
    """A device-resident graph index (one GPU)."""

    def __init__(self, graph, storage=("f32",), device=0):
        lib = _lib.load()
        self._graph_keepalive = graph
        d = _lib.IndexDesc()
        d.num_vectors = graph.n
        d.dim = graph.dim
        d.max_degree = graph.max_degree
        d.vectors = graph.vectors.ctypes.data
        d.vector_stride = graph.vectors.strides[0] // 4
        d.links = graph.links.ctypes.data
        d.link_stride = graph.links.strides[0] // 4
        d.ids_offset = graph.ids_offset
        d.entry_point = graph.entry_point
        d.labels = graph.labels.ctypes.data if graph.labels is not None else None
        d.storage = storage_mask(storage)
        d.device = int(device)
        h = ctypes.c_void_p()
        _lib.check(lib.falcon_index_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self.device = int(device)
        self.dim = graph.dim
        self.n = graph.n

    @classmethod
    def load_fpga(cls, index_dir, graph_type, dim, storage=("f32",), device=0):
        lib = _lib.load()
        obj = cls.__new__(cls)
        h = ctypes.c_void_p()
        _lib.check(lib.falcon_index_load_fpga(index_dir.encode(), graph_type.encode(), int(dim),
                                              storage_mask(storage), int(device), ctypes.byref(h)))
        obj._h = h
        obj._graph_keepalive = None
        obj.device = int(device)
        info = obj.info()
        obj.dim, obj.n = info.dim, info.num_vectors
        return obj

    def info(self):
        inf = _lib.IndexInfo()
        _lib.check(_lib.load().falcon_index_info_get(self._h, ctypes.byref(inf)))
        return inf

    def storage(self, which="f32"):
        """Copy a resident storage array back: f32 [n, dpad] float32, bf16
        [n, dpad] uint16 codes, fp8 ([n, dpad] uint8 codes, [n] float32 scales)."""
        inf = self.info()
        n, dp = inf.num_vectors, inf.dim_padded
        lib = _lib.load()
        if which == "f32":
            out = np.empty((n, dp), dtype=np.float32)
        elif which == "bf16":
            out = np.empty((n, dp), dtype=np.uint16)
        elif which == "fp8":
            out = np.empty(n * dp + 4 * n, dtype=np.uint8)
        else:
            raise ValueError(which)
        _lib.check(lib.falcon_index_copy_storage(self._h, _STORE[which], out.ctypes.data, out.nbytes))
        if which == "fp8":
            return out[:n * dp].reshape(n, dp), out[n * dp:].view(np.float32).copy()
        return out

    def set_upper_layers(self, upper):
        """Attach HNSW upper layers (formats.UpperLayers); afterwards searches
        without entry points start from the greedy descent's entry."""
        rows = np.ascontiguousarray(upper.rows, dtype=np.int32)
        levels = np.ascontiguousarray(upper.levels, dtype=np.int32)
        starts = np.ascontiguousarray(upper.row_start, dtype=np.int64)
        d = _lib.UpperLayersDesc()
        d.max_level, d.max_degree, d.entry_point, d.ids_offset = upper.max_level, upper.max_degree, upper.entry, 1
        d.num_rows, d.row_stride = rows.shape[0], rows.shape[1]
        d.levels, d.row_start, d.rows = levels.ctypes.data, starts.ctypes.data, rows.ctypes.data
        _lib.check(_lib.load().falcon_index_set_upper_layers(self._h, ctypes.byref(d)))

    def descend(self, queries, stream=None):
        """Base-layer entry point per query from the upper-layer descent, and
        the number of upper rows expanded: (entries, hops), numpy for host
        queries, torch for device queries."""
        lib = _lib.load()
        if _is_torch_cuda(queries):
            import torch
            q = queries.contiguous().float()
            ent = torch.empty(q.shape[0], dtype=torch.int32, device=q.device)
            hops = torch.empty(q.shape[0], dtype=torch.int32, device=q.device)
            s = stream if stream is not None else torch.cuda.current_stream(q.device).cuda_stream
            _lib.check(lib.falcon_descend(self._h, q.data_ptr(), q.shape[0], q.stride(0), ent.data_ptr(),
                                          hops.data_ptr(), _lib.MEM_DEVICE, ctypes.c_void_p(s)))
            return ent, hops
        q = np.ascontiguousarray(queries, dtype=np.float32)
        ent = np.empty(q.shape[0], dtype=np.int32)
        hops = np.empty(q.shape[0], dtype=np.int32)
        _lib.check(lib.falcon_descend(self._h, q.ctypes.data, q.shape[0], q.shape[1], ent.ctypes.data,
                                      hops.ctypes.data, _lib.MEM_HOST, stream))
        return ent, hops

    def close(self):
        if getattr(self, "_h", None):
            # refused while a server holds the index: keep the handle
            _lib.check(_lib.load().falcon_index_free(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def search(self, queries, k=10, ef=64, mc=1, mg=1, cand_queue_size=32, bloom_bits=16, hash_seed=1,
               mode="inter", channels=4, precision="f32", rerank=False, max_hops=0, entry_points=None,
               per_query=None, out_stride=None, stream=None, out=None):
        """Search host queries [nq, dim] (numpy) or device queries (torch CUDA tensor).

        per_query: optional list of dicts or SearchParams, one per query, or
        a params_array (mixed k/ef/mc in one launch; host or device queries).  Returns (ids, dists, hops, visited) with
        ids/dists [nq, out_stride] best-first (out_stride = max k by default).
        out: result arrays (ids, dists, hops, visited) to write into and
        return, reused across calls: numpy arrays for host queries (e.g.
        pinned_results(nq, out_stride)), CUDA tensors on the queries' device
        for device queries (device_results(nq, out_stride)).
        """
        lib = _lib.load()
        if per_query is not None:
            arr = per_query if isinstance(per_query, ctypes.Array) else params_array(per_query)
            params, pq, kmax = arr, 1, max_k(arr)
        else:
            params, pq = make_params(k, ef, mc, mg, cand_queue_size, bloom_bits, hash_seed, mode, channels,
                                     precision, rerank, max_hops), 0
            kmax = params.k
        ostride = int(out_stride or kmax)
        if _is_torch_cuda(queries):
            return self._search_device(queries, params, pq, ostride, entry_points, stream, out)
        q = np.ascontiguousarray(queries, dtype=np.float32)
        if q.ndim != 2 or q.shape[1] != self.dim:
            raise ValueError("queries must be [nq, %d]" % self.dim)
        nq = q.shape[0]
        if out is not None:
            ids, dists, hops, vis = out
            for a, shape, dt in ((ids, (nq, ostride), np.int32), (dists, (nq, ostride), np.float32),
                                 (hops, (nq,), np.int32), (vis, (nq,), np.int32)):
                if a.shape != shape or a.dtype != dt or not a.flags.c_contiguous:
                    raise ValueError("out arrays must be C-contiguous %s %s" % (shape, np.dtype(dt).name))
        else:
            ids = np.empty((nq, ostride), dtype=np.int32)
            dists = np.empty((nq, ostride), dtype=np.float32)
            hops = np.empty(nq, dtype=np.int32)
            vis = np.empty(nq, dtype=np.int32)
        ep = None
        if entry_points is not None:
            ep = np.ascontiguousarray(entry_points, dtype=np.int32)
        pptr = ctypes.cast(params, ctypes.POINTER(_lib.SearchParams)) if pq else ctypes.byref(params)
        rc = lib.falcon_search(self._h, q.ctypes.data, nq, q.shape[1], ep.ctypes.data if ep is not None else None,
                               pptr, pq, ids.ctypes.data, dists.ctypes.data, ostride, hops.ctypes.data,
                               vis.ctypes.data, _lib.MEM_HOST, stream)
        _lib.check(rc)
        return SearchResult(ids, dists, hops, vis, rc)

    def search_trace(self, queries, cand_capacity=4096, capacity=65536, k=10, ef=64, mc=1, mg=1,
                     cand_queue_size=32, bloom_bits=16, hash_seed=1, max_hops=0, entry_points=None, stream=None):
        """FP32 inter-query search with the traversal trace (falcon_search_trace)
        on host queries.  Returns (SearchResult, Trace)."""
        lib = _lib.load()
        params = make_params(k, ef, mc, mg, cand_queue_size, bloom_bits, hash_seed, "inter", 4, "f32", False,
                             max_hops)
        q = np.ascontiguousarray(queries, dtype=np.float32)
        nq = q.shape[0]
        ids = np.empty((nq, k), dtype=np.int32)
        dists = np.empty((nq, k), dtype=np.float32)
        hops = np.empty(nq, dtype=np.int32)
        vis = np.empty(nq, dtype=np.int32)
        cd = np.zeros((nq, cand_capacity), dtype=np.float32)
        cn = np.zeros((nq, cand_capacity), dtype=np.int32)
        td = np.zeros((nq, capacity), dtype=np.float32)
        ti = np.zeros((nq, capacity), dtype=np.int32)
        cnt = np.zeros((nq, 3), dtype=np.int32)
        ep = None if entry_points is None else np.ascontiguousarray(entry_points, dtype=np.int32)
        rc = lib.falcon_search_trace(self._h, q.ctypes.data, nq, q.shape[1], ep.ctypes.data if ep is not None else None,
                                     ctypes.byref(params), ids.ctypes.data, dists.ctypes.data, k, hops.ctypes.data,
                                     vis.ctypes.data, cd.ctypes.data, cn.ctypes.data, cand_capacity, td.ctypes.data,
                                     ti.ctypes.data, capacity, cnt.ctypes.data, _lib.MEM_HOST, stream)
        _lib.check(rc)
        return SearchResult(ids, dists, hops, vis, rc), Trace(cd, cn, td, ti, cnt)

    def _search_device(self, queries, params, pq, ostride, entry_points, stream, out=None):
        import torch
        lib = _lib.load()
        q = queries.contiguous().float()
        nq = q.shape[0]
        dev = q.device
        if out is not None:
            ids, dists, hops, vis = out
            for a, shape, dt in ((ids, (nq, ostride), torch.int32), (dists, (nq, ostride), torch.float32),
                                 (hops, (nq,), torch.int32), (vis, (nq,), torch.int32)):
                if (not isinstance(a, torch.Tensor) or a.device != dev or tuple(a.shape) != shape or a.dtype != dt
                        or not a.is_contiguous()):
                    raise ValueError("out tensors must be contiguous %s %s on %s" % (shape, dt, dev))
        else:
            ids = torch.empty((nq, ostride), dtype=torch.int32, device=dev)
            dists = torch.empty((nq, ostride), dtype=torch.float32, device=dev)
            hops = torch.empty(nq, dtype=torch.int32, device=dev)
            vis = torch.empty(nq, dtype=torch.int32, device=dev)
        ep = None
        if entry_points is not None:
            ep = entry_points.to(device=dev, dtype=torch.int32).contiguous()
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        pptr = ctypes.cast(params, ctypes.POINTER(_lib.SearchParams)) if pq else ctypes.byref(params)
        rc = lib.falcon_search(self._h, q.data_ptr(), nq, q.stride(0), ep.data_ptr() if ep is not None else None,
                               pptr, pq, ids.data_ptr(), dists.data_ptr(), ostride, hops.data_ptr(),
                               vis.data_ptr(), _lib.MEM_DEVICE, ctypes.c_void_p(s))
        _lib.check(rc)
        return SearchResult(ids, dists, hops, vis, rc)


def pinned_results(nq, out_stride):
    """(ids, dists, hops, visited) arrays in page-locked host memory, for
    search(..., out=...): the device-to-host copies of a host-memory search
    then run at full link bandwidth and touch no fresh pages (the reference's
    host likewise allocates its result buffers once)."""
    import torch
    return (torch.empty((nq, out_stride), dtype=torch.int32, pin_memory=True).numpy(),
            torch.empty((nq, out_stride), dtype=torch.float32, pin_memory=True).numpy(),
            torch.empty(nq, dtype=torch.int32, pin_memory=True).numpy(),
            torch.empty(nq, dtype=torch.int32, pin_memory=True).numpy())


def device_results(nq, out_stride, device=0):
    """(ids, dists, hops, visited) CUDA tensors for search(..., out=...) on
    device queries: a caller that searches small batches in a loop allocates
    its result buffers once instead of four times per call."""
    import torch
    return (torch.empty((nq, out_stride), dtype=torch.int32, device=device),
            torch.empty((nq, out_stride), dtype=torch.float32, device=device),
            torch.empty(nq, dtype=torch.int32, device=device),
            torch.empty(nq, dtype=torch.int32, device=device))


def _is_torch_cuda(x):
    try:
        import torch
    except ImportError:
        return False
    return isinstance(x, torch.Tensor) and x.is_cuda


def vadd(query_vectors_padded, entry_point_ids, db_vectors_ref, links_ref, num_db_vec, dim, ef=64,
         candidate_queue_runtime_size=32, max_cand_batch_size=1, max_async_stage_num=1,
         runtime_n_bucket_addr_bits=16, hash_seed=1, max_bloom_out_burst_size=16, max_link_num_base=64,
         query_batch_size=None, device=0):
    """The reference kernel's argument list (vadd.cpp:11-95) on reference-layout host buffers."""
    lib = _lib.load()
    qv = np.ascontiguousarray(query_vectors_padded, dtype=np.float32)
    nq = qv.shape[0]
    ep = np.ascontiguousarray(entry_point_ids, dtype=np.int32)
    out_id = np.empty((nq, ef), dtype=np.int32)
    out_dist = np.empty((nq, ef), dtype=np.float32)
    mem_debug = np.empty((nq, 2), dtype=np.int32)
    dv = np.ascontiguousarray(db_vectors_ref)
    lk = np.ascontiguousarray(links_ref)
    rc = lib.falcon_vadd(nq, int(query_batch_size or max(nq, 1)), ef, candidate_queue_runtime_size,
                         max_cand_batch_size, max_async_stage_num, runtime_n_bucket_addr_bits, hash_seed,
                         max_bloom_out_burst_size, max_link_num_base, dim, num_db_vec, ep.ctypes.data,
                         qv.ctypes.data, dv.ctypes.data, lk.ctypes.data, out_id.ctypes.data, out_dist.ctypes.data,
                         mem_debug.ctypes.data, device)
    _lib.check(rc)
    return out_id, out_dist, mem_debug


__all__ = ["FalconIndex", "Graph", "make_params", "params_array", "vadd", "storage_mask"]
