"""TEST INFRASTRUCTURE ONLY: Python access to the parity oracle.

  search(...)          the C restatement (oracle/falcon_oracle.c)
  ref_inter_search(...) the reference's own v1.3 HLS kernel compiled as C++
                        (oracle/_ref/libfalcon_ref_d{D}.so)
  Hnsw                 the reference's vendored hnswlib (oracle/_ref/libhnswlib_ref.so)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm use this module.  The product library never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

F32, BF16, FP8 = 0, 1, 2


class FoGraph(ctypes.Structure):
    _fields_ = [
        ("vectors", ctypes.c_void_p),
        ("scales", ctypes.c_void_p),
        ("elem", ctypes.c_int),
        ("vec_stride", ctypes.c_int64),
        ("vectors_f32", ctypes.c_void_p),
        ("vec_stride_f32", ctypes.c_int64),
        ("links", ctypes.c_void_p),
        ("link_stride", ctypes.c_int64),
        ("ids_offset", ctypes.c_int),
        ("max_degree", ctypes.c_int),
        ("dim", ctypes.c_int),
        ("dpad", ctypes.c_int),
        ("n", ctypes.c_int64),
    ]


class FoUpper(ctypes.Structure):
    _fields_ = [
        ("rows", ctypes.c_void_p),
        ("row_stride", ctypes.c_int64),
        ("ids_offset", ctypes.c_int),
        ("row_start", ctypes.c_void_p),
        ("levels", ctypes.c_void_p),
        ("max_level", ctypes.c_int),
        ("entry", ctypes.c_int),
    ]


class FoParams(ctypes.Structure):
    _fields_ = [
        ("k", ctypes.c_int), ("ef", ctypes.c_int), ("mc", ctypes.c_int), ("mg", ctypes.c_int),
        ("cand_queue_size", ctypes.c_int), ("bloom_bits", ctypes.c_int), ("hash_seed", ctypes.c_uint32),
        ("mode", ctypes.c_int), ("channels", ctypes.c_int), ("rerank", ctypes.c_int), ("max_hops", ctypes.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        p = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(p):
            import build_oracle   # noqa: F401  (oracle/ on sys.path)
            build_oracle.build_oracle()
        _lib = ctypes.CDLL(p)
        _lib.fo_search.restype = ctypes.c_int
        _lib.fo_search.argtypes = [ctypes.POINTER(FoGraph), ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _lib.fo_murmur2_keylen4.restype = ctypes.c_uint32
        _lib.fo_murmur2_keylen4.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        _lib.fo_fp8e4m3_to_f32.restype = ctypes.c_float
        _lib.fo_fp8e4m3_to_f32.argtypes = [ctypes.c_uint8]
        _lib.fo_queue_insert_sort.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        _lib.fo_bloom_stream.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p]
        _lib.fo_l2_batch.argtypes = [ctypes.POINTER(FoGraph), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_void_p]
        _lib.fo_search_trace.restype = ctypes.c_int
        _lib.fo_search_trace.argtypes = [ctypes.POINTER(FoGraph), ctypes.POINTER(FoParams), ctypes.c_void_p,
                                         ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int] + \
            [ctypes.c_void_p] * 6 + [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_int]
        _lib.fo_descend.restype = ctypes.c_int
        _lib.fo_descend.argtypes = [ctypes.POINTER(FoGraph), ctypes.POINTER(FoUpper), ctypes.c_void_p,
                                    ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    return _lib


def pad16(d):
    return (d + 15) // 16 * 16


class OracleGraph:
    """Keeps the arrays alive and builds the fo_graph view.

    vectors_f32: [n, dim] float32; links: reference layout rows.
    elem/stored: the traversal storage (F32, or BF16 uint16 codes [n, dpad],
    or FP8 uint8 codes [n, dpad] + scales [n])."""

    def __init__(self, vectors_f32, links, max_degree, ids_offset=16, elem=F32, stored=None, scales=None):
        n, dim = vectors_f32.shape
        self.dim, self.dpad, self.n = dim, pad16(dim), n
        v = np.zeros((n, self.dpad), dtype=np.float32)
        v[:, :dim] = vectors_f32
        self.v32 = v
        self.links = np.ascontiguousarray(links, dtype=np.int32)
        self.stored = v if elem == F32 else np.ascontiguousarray(stored)
        self.scales = None if scales is None else np.ascontiguousarray(scales, dtype=np.float32)
        g = FoGraph()
        g.vectors = self.stored.ctypes.data
        g.scales = self.scales.ctypes.data if self.scales is not None else None
        g.elem = elem
        g.vec_stride = self.stored.shape[1]
        g.vectors_f32 = v.ctypes.data
        g.vec_stride_f32 = self.dpad
        g.links = self.links.ctypes.data
        g.link_stride = self.links.shape[1]
        g.ids_offset = ids_offset
        g.max_degree = max_degree
        g.dim = dim
        g.dpad = self.dpad
        g.n = n
        self.g = g


def make_params(k=10, ef=64, mc=1, mg=1, cand_queue_size=32, bloom_bits=16, hash_seed=1, mode="inter",
                channels=4, rerank=False, max_hops=0, precision=None):
    """precision is accepted for symmetry with the product's parameters; the
    traversal storage is chosen by the OracleGraph the search runs on."""
    p = FoParams()
    p.k, p.ef, p.mc, p.mg = k, ef, mc, mg
    p.cand_queue_size, p.bloom_bits, p.hash_seed = cand_queue_size, bloom_bits, hash_seed
    p.mode = 0 if mode == "inter" else 1
    p.channels, p.rerank, p.max_hops = channels, 1 if rerank else 0, max_hops
    return p


def search(og, queries, entries, params, out_stride=None, threads=None):
    """params: one FoParams or a list (one per query).  Returns ids, dists, hops, visited, status."""
    q = np.ascontiguousarray(queries, dtype=np.float32)
    nq = q.shape[0]
    e = np.ascontiguousarray(np.broadcast_to(np.asarray(entries, dtype=np.int32), (nq,)))
    if isinstance(params, FoParams):
        parr, stride, kmax = params, 0, params.k
    else:
        parr = (FoParams * nq)(*params)
        stride, kmax = 1, max(p.k for p in params)
    os_ = out_stride or kmax
    ids = np.empty((nq, os_), dtype=np.int32)
    d = np.empty((nq, os_), dtype=np.float32)
    hops = np.empty(nq, dtype=np.int32)
    vis = np.empty(nq, dtype=np.int32)
    threads = threads or min(32, os.cpu_count() or 1)
    rc = lib().fo_search(ctypes.byref(og.g), ctypes.byref(parr) if stride == 0 else parr, stride, q.ctypes.data,
                         q.shape[1], e.ctypes.data, nq, os_, ids.ctypes.data, d.ctypes.data, hops.ctypes.data,
                         vis.ctypes.data, threads)
    if rc < 0:
        raise ValueError("oracle rejected arguments: %d" % rc)
    return ids, d, hops, vis, rc


def descend(og, upper, queries):
    """HNSW upper-layer greedy descent (fo_descend).  upper: an object with
    max_level, entry, levels [n] int32, row_start [n] int64 and rows
    [num_rows, 1 + max_degree] int32 (count, then ids), as
    falcon_b200.formats.UpperLayers.  Returns (entries, upper hops)."""
    q = np.ascontiguousarray(queries, dtype=np.float32)
    rows = np.ascontiguousarray(upper.rows, dtype=np.int32)
    starts = np.ascontiguousarray(upper.row_start, dtype=np.int64)
    levels = np.ascontiguousarray(upper.levels, dtype=np.int32)
    u = FoUpper()
    u.rows = rows.ctypes.data
    u.row_stride = rows.shape[1]
    u.ids_offset = 1
    u.row_start = starts.ctypes.data
    u.levels = levels.ctypes.data
    u.max_level = int(upper.max_level)
    u.entry = int(upper.entry)
    nq = q.shape[0]
    ent = np.empty(nq, dtype=np.int32)
    hops = np.empty(nq, dtype=np.int32)
    rc = lib().fo_descend(ctypes.byref(og.g), ctypes.byref(u), q.ctypes.data, nq, q.shape[1], ent.ctypes.data,
                          hops.ctypes.data)
    if rc < 0:
        raise MemoryError("oracle descent failed")
    return ent, hops


def search_trace(og, queries, entries, params, cand_cap, cap, threads=None):
    """Inter-query search with the traversal trace (fo_search_trace).  Returns
    ids, dists, hops, visited, and the trace: cand_d [nq, cand_cap],
    cand_n [nq, cand_cap], d [nq, cap], id [nq, cap], counts [nq, 3]
    (popped incl. entry, expanded, computed distances)."""
    q = np.ascontiguousarray(queries, dtype=np.float32)
    nq = q.shape[0]
    e = np.ascontiguousarray(np.broadcast_to(np.asarray(entries, dtype=np.int32), (nq,)))
    k = params.k
    ids = np.empty((nq, k), dtype=np.int32)
    d = np.empty((nq, k), dtype=np.float32)
    hops = np.empty(nq, dtype=np.int32)
    vis = np.empty(nq, dtype=np.int32)
    cd = np.zeros((nq, cand_cap), dtype=np.float32)
    cn = np.zeros((nq, cand_cap), dtype=np.int32)
    td = np.zeros((nq, cap), dtype=np.float32)
    ti = np.zeros((nq, cap), dtype=np.int32)
    cnt = np.zeros((nq, 3), dtype=np.int32)
    threads = threads or min(32, os.cpu_count() or 1)
    rc = lib().fo_search_trace(ctypes.byref(og.g), ctypes.byref(params), q.ctypes.data, q.shape[1], e.ctypes.data, nq,
                               k, ids.ctypes.data, d.ctypes.data, hops.ctypes.data, vis.ctypes.data, cd.ctypes.data,
                               cn.ctypes.data, cand_cap, td.ctypes.data, ti.ctypes.data, cap, cnt.ctypes.data, threads)
    if rc < 0:
        raise ValueError("oracle rejected arguments: %d" % rc)
    return ids, d, hops, vis, (cd, cn, td, ti, cnt)


def murmur2(key, seed):
    return int(lib().fo_murmur2_keylen4(key & 0xffffffff, seed & 0xffffffff))


def fp8_to_f32(code):
    return float(lib().fo_fp8e4m3_to_f32(code))


def queue_insert_sort(values, ids, n, v15=False):
    """Insert a stream into an n-slot systolic queue, then sort; returns the
    queue best-first (ids, dists), like the reference's unit test kernel."""
    vals = np.ascontiguousarray(values, dtype=np.float32)
    iv = np.ascontiguousarray(ids, dtype=np.int32)
    d = np.empty(n, dtype=np.float32)
    i = np.empty(n, dtype=np.int32)
    lib().fo_queue_insert_sort(d.ctypes.data, i.ctypes.data, n, vals.ctypes.data, iv.ctypes.data, len(vals),
                               1 if v15 else 0)
    return i[::-1].copy(), d[::-1].copy()


def bloom_stream(keys, bits=16, seed=1):
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    out = np.empty(len(k), dtype=np.uint8)
    lib().fo_bloom_stream(k.ctypes.data, len(k), bits, seed, out.ctypes.data)
    return out


def l2_batch(og, query, ids):
    q = np.ascontiguousarray(query, dtype=np.float32)
    i = np.ascontiguousarray(ids, dtype=np.int32)
    out = np.empty(len(i), dtype=np.float32)
    lib().fo_l2_batch(ctypes.byref(og.g), q.ctypes.data, i.ctypes.data, len(i), out.ctypes.data)
    return out


# ---------------------------------------------------------------------------
# Reference harness (the reference's own HLS kernel code run as C++)
# ---------------------------------------------------------------------------
_ref_libs = {}


def ref_available(dim):
    return os.path.exists(os.path.join(REF_DIR, "libfalcon_ref_d%d.so" % dim))


def _ref_lib(dim):
    if dim not in _ref_libs:
        p = os.path.join(REF_DIR, "libfalcon_ref_d%d.so" % dim)
        L = ctypes.CDLL(p)
        L.ref_inter_search.restype = ctypes.c_int
        L.ref_inter_search.argtypes = [ctypes.c_int] * 6 + [ctypes.c_uint, ctypes.c_int, ctypes.c_int] + \
            [ctypes.c_void_p] * 7
        _ref_libs[dim] = L
    return _ref_libs[dim]


def ref_trace_available():
    return os.path.exists(os.path.join(REF_DIR, "libfalcon_ref_trace_d128.so"))


def ref_inter_search_trace(vectors, links_ref, max_degree, queries, entries, ef=64, cand_queue_size=32, mc=1, mg=1,
                           bloom_bits=16, hash_seed=1, burst=16):
    """The reference's trace kernel (eval_trace_FPGA_inter_query_v1.3, D = 128)
    on reference-layout data.  Returns ids, dists, hops, visited and per query
    the lists (cand_d, cand_n, d, ids) cut from its flat -1 ... -2 streams."""
    n, dim = vectors.shape
    if dim != 128:
        raise ValueError("the trace harness is built for D = 128")
    p = os.path.join(REF_DIR, "libfalcon_ref_trace_d128.so")
    L = ctypes.CDLL(p)
    L.ref_inter_search_trace.restype = ctypes.c_int
    L.ref_inter_search_trace.argtypes = [ctypes.c_int] * 6 + [ctypes.c_uint, ctypes.c_int, ctypes.c_int] + \
        [ctypes.c_void_p] * 11
    db = np.zeros((n, 128 + 16), dtype=np.float32)
    db[:, :dim] = vectors
    q = np.ascontiguousarray(queries, dtype=np.float32)
    nq = len(q)
    e = np.ascontiguousarray(np.broadcast_to(np.asarray(entries, dtype=np.int32), (nq,)))
    lk = np.ascontiguousarray(links_ref, dtype=np.int32)
    oid = np.empty((nq, ef), dtype=np.int32)
    od = np.empty((nq, ef), dtype=np.float32)
    dbg = np.empty((nq, 2), dtype=np.int32)
    cap = nq * (n + 2)          # visited <= n and hops <= visited + 1 per query
    cd = np.zeros(cap, dtype=np.float32)
    cn = np.zeros(cap, dtype=np.int32)
    td = np.zeros(cap, dtype=np.float32)
    ti = np.zeros(cap, dtype=np.int32)
    rc = L.ref_inter_search_trace(nq, ef, cand_queue_size, mc, mg, bloom_bits, hash_seed, burst, max_degree,
                                  e.ctypes.data, q.ctypes.data, db.ctypes.data, lk.ctypes.data, oid.ctypes.data,
                                  od.ctypes.data, dbg.ctypes.data, cd.ctypes.data, cn.ctypes.data, td.ctypes.data,
                                  ti.ctypes.data)
    if rc != 0:
        raise ValueError("reference harness rejected arguments")

    def split(a, b):
        out, i = [], 0
        for _ in range(nq):
            assert a[i] == -1 and b[i] == -1
            j = i + 1
            while not (a[j] == -2 and b[j] == -2):
                j += 1
            out.append((a[i + 1:j].copy(), b[i + 1:j].copy()))
            i = j + 1
        return out
    cand = split(cd, cn)
    dist = split(td, ti)
    trace = [(c[0], c[1], d_[0], d_[1]) for c, d_ in zip(cand, dist)]
    return oid, od, dbg[:, 0].copy(), dbg[:, 1].copy(), trace


def ref_inter_search(vectors, links_ref, max_degree, queries, entries, ef=64, cand_queue_size=32, mc=1, mg=1,
                     bloom_bits=16, hash_seed=1, burst=16):
    """Run the reference kernel pipeline (one channel) on reference-layout data."""
    n, dim = vectors.shape
    L = _ref_lib(dim)
    dp = pad16(dim)
    db = np.zeros((n, dp + 16), dtype=np.float32)
    db[:, :dim] = vectors
    q = np.zeros((len(queries), dp), dtype=np.float32)
    q[:, :dim] = queries
    e = np.ascontiguousarray(np.broadcast_to(np.asarray(entries, dtype=np.int32), (len(queries),)))
    lk = np.ascontiguousarray(links_ref, dtype=np.int32)
    nq = len(queries)
    oid = np.empty((nq, ef), dtype=np.int32)
    od = np.empty((nq, ef), dtype=np.float32)
    dbg = np.empty((nq, 2), dtype=np.int32)
    rc = L.ref_inter_search(nq, ef, cand_queue_size, mc, mg, bloom_bits, hash_seed, burst, max_degree, e.ctypes.data,
                            q.ctypes.data, db.ctypes.data, lk.ctypes.data, oid.ctypes.data, od.ctypes.data,
                            dbg.ctypes.data)
    if rc != 0:
        raise ValueError("reference harness rejected arguments")
    return oid, od, dbg[:, 0].copy(), dbg[:, 1].copy()


def ref_intra_available(dim, channels):
    return os.path.exists(os.path.join(REF_DIR, "libfalcon_ref_intra_d%d_c%d.so" % (dim, channels)))


def ref_intra_search(vectors, links_ref, max_degree, queries, entries, channels, ef=64, cand_queue_size=32, mc=1,
                     mg=1, bloom_bits=16, hash_seed=1, burst=16):
    """Run the reference's intra-query v1.5 kernel pipeline (N channels, the
    nodes spread round robin over them) on node-ordered reference-layout data.
    Returns ids, dists, hops (v1.5 reports no visited count)."""
    n, dim = vectors.shape
    key = ("intra", dim, channels)
    if key not in _ref_libs:
        L = ctypes.CDLL(os.path.join(REF_DIR, "libfalcon_ref_intra_d%d_c%d.so" % (dim, channels)))
        L.ref_intra_search.restype = ctypes.c_int
        L.ref_intra_search.argtypes = [ctypes.c_int] * 6 + [ctypes.c_uint, ctypes.c_int, ctypes.c_int,
                                                            ctypes.c_int64] + [ctypes.c_void_p] * 7
        _ref_libs[key] = L
    L = _ref_libs[key]
    dp = pad16(dim)
    db = np.zeros((n, dp + 16), dtype=np.float32)
    db[:, :dim] = vectors
    q = np.zeros((len(queries), dp), dtype=np.float32)
    q[:, :dim] = queries
    nq = len(queries)
    e = np.ascontiguousarray(np.broadcast_to(np.asarray(entries, dtype=np.int32), (nq,)))
    lk = np.ascontiguousarray(links_ref, dtype=np.int32)
    oid = np.empty((nq, ef), dtype=np.int32)
    od = np.empty((nq, ef), dtype=np.float32)
    dbg = np.empty((nq, 1), dtype=np.int32)
    rc = L.ref_intra_search(nq, ef, cand_queue_size, mc, mg, bloom_bits, hash_seed, burst, max_degree, n,
                            e.ctypes.data, q.ctypes.data, db.ctypes.data, lk.ctypes.data, oid.ctypes.data,
                            od.ctypes.data, dbg.ctypes.data)
    if rc != 0:
        raise ValueError("reference harness rejected arguments")
    return oid, od, dbg[:, 0].copy()


# ---------------------------------------------------------------------------
# Reference hnswlib
# ---------------------------------------------------------------------------
class Hnsw:
    def __init__(self, handle, dim):
        self.h, self.dim = handle, dim

    _lib_cache = None

    @staticmethod
    def isa():
        """The ISA level of the hnswlib build this CPU runs: "x86-64-v4"
        (AVX-512) when /proc/cpuinfo lists avx512 f/bw/cd/dq/vl and that
        build exists, else "avx2"."""
        try:
            flags = set()
            with open("/proc/cpuinfo") as f:
                for line in f:
                    if line.startswith("flags"):
                        flags = set(line.split(":", 1)[1].split())
                        break
        except OSError:
            flags = set()
        v4 = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags
        if v4 and os.path.exists(os.path.join(REF_DIR, "libhnswlib_ref_v4.so")):
            return "x86-64-v4"
        return "avx2"

    @staticmethod
    def cpu_model():
        try:
            with open("/proc/cpuinfo") as f:
                for line in f:
                    if line.startswith("model name"):
                        return line.split(":", 1)[1].strip()
        except OSError:
            pass
        return "unknown"

    @staticmethod
    def _L():
        if Hnsw._lib_cache is not None:
            return Hnsw._lib_cache
        name = "libhnswlib_ref_v4.so" if Hnsw.isa() == "x86-64-v4" else "libhnswlib_ref.so"
        L = ctypes.CDLL(os.path.join(REF_DIR, name))
        L.hnsw_build.restype = ctypes.c_void_p
        L.hnsw_build.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.hnsw_from_graph.restype = ctypes.c_void_p
        L.hnsw_from_graph.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_int]
        L.hnsw_info.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4
        L.hnsw_export_level0.argtypes = [ctypes.c_void_p] * 4
        L.hnsw_search.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.hnsw_free.argtypes = [ctypes.c_void_p]
        L.hnsw_save.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.hnsw_upper_rows.restype = ctypes.c_int64
        L.hnsw_upper_rows.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.hnsw_export_upper.argtypes = [ctypes.c_void_p] * 4
        L.hnsw_descend.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p]
        L.hnsw_set_upper.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        Hnsw._lib_cache = L
        return L

    @classmethod
    def available(cls):
        return os.path.exists(os.path.join(REF_DIR, "libhnswlib_ref.so"))

    @classmethod
    def build(cls, vectors, M, ef_construction, seed):
        v = np.ascontiguousarray(vectors, dtype=np.float32)
        h = cls._L().hnsw_build(v.shape[0], v.shape[1], M, ef_construction, seed, v.ctypes.data)
        obj = cls(h, v.shape[1])
        obj._keep = v
        return obj

    @classmethod
    def from_graph(cls, vectors, adjacency, entry):
        v = np.ascontiguousarray(vectors, dtype=np.float32)
        adj = np.ascontiguousarray(adjacency, dtype=np.int32)
        counts = (adj >= 0).sum(1).astype(np.int32)
        h = cls._L().hnsw_from_graph(v.shape[0], v.shape[1], adj.shape[1], v.ctypes.data, adj.ctypes.data,
                                     counts.ctypes.data, int(entry))
        obj = cls(h, v.shape[1])
        obj._keep = (v, adj, counts)
        return obj

    def set_upper(self, upper):
        """Give an index made by from_graph the HNSW upper layers of a
        formats.UpperLayers (rows: count at [0], ids from [1]); searchKnn then
        descends them first, as in an index hnswlib built itself."""
        levels = np.ascontiguousarray(upper.levels, dtype=np.int32)
        starts = np.ascontiguousarray(upper.row_start, dtype=np.int64)
        rows = np.ascontiguousarray(upper.rows, dtype=np.int32)
        rc = self._L().hnsw_set_upper(self.h, levels.ctypes.data, starts.ctypes.data, rows.ctypes.data,
                                      rows.shape[1], 1, int(upper.max_level), int(upper.entry))
        if rc != 0:
            raise ValueError("upper-layer list longer than hnswlib's maxM_")
        self._keep_upper = (levels, starts, rows)

    def search_mixed(self, queries, ks, efs, threads, out_stride=None):
        """searchKnn with per-query k and ef: the queries are grouped by
        (ef, k) and each group is searched with setEf(ef) over all threads.
        Returns labels / distances [nq, out_stride] (-1 / 1e20 padded)."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        ks, efs = np.asarray(ks), np.asarray(efs)
        w = int(out_stride or ks.max())
        lab = np.full((len(q), w), -1, dtype=np.int64)
        d = np.full((len(q), w), 1e20, dtype=np.float32)
        for ef in np.unique(efs):
            for k in np.unique(ks):
                sel = np.nonzero((efs == ef) & (ks == k))[0]
                if sel.size:
                    l_, d_ = self.search(q[sel], int(k), int(ef), threads)
                    lab[sel, :k], d[sel, :k] = l_, d_
        return lab, d

    def level0(self):
        L = self._L()
        n = ctypes.c_int64()
        md = ctypes.c_int()
        ep = ctypes.c_int()
        ml = ctypes.c_int()
        L.hnsw_info(self.h, ctypes.byref(n), ctypes.byref(md), ctypes.byref(ep), ctypes.byref(ml))
        links = np.empty((n.value, md.value), dtype=np.int32)
        counts = np.empty(n.value, dtype=np.int32)
        labels = np.empty(n.value, dtype=np.int32)
        L.hnsw_export_level0(self.h, links.ctypes.data, counts.ctypes.data, labels.ctypes.data)
        return links, counts, labels, ep.value, ml.value

    def save(self, path):
        """hnswlib's own saveIndex."""
        self._L().hnsw_save(self.h, path.encode())

    def upper(self):
        """(max_level, entry, max_m, levels [n], row_start [n], rows [num_rows, 1 + max_m]) through
        hnswlib's accessors."""
        L = self._L()
        links, counts, labels, ep, ml = self.level0()
        n = links.shape[0]
        mm = ctypes.c_int()
        nrows = L.hnsw_upper_rows(self.h, ctypes.byref(mm))
        levels = np.empty(n, dtype=np.int32)
        starts = np.empty(n, dtype=np.int64)
        rows = np.zeros((max(nrows, 1), 1 + mm.value), dtype=np.int32)
        L.hnsw_export_upper(self.h, levels.ctypes.data, starts.ctypes.data, rows.ctypes.data)
        return ml, ep, mm.value, levels, starts, rows

    def descend(self, queries):
        """Base-layer entry per query from hnswlib's greedy upper-layer search."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        out = np.empty(len(q), dtype=np.int32)
        self._L().hnsw_descend(self.h, q.ctypes.data, len(q), self.dim, out.ctypes.data)
        return out

    def search(self, queries, k, ef, threads):
        q = np.ascontiguousarray(queries, dtype=np.float32)
        lab = np.empty((len(q), k), dtype=np.int64)
        d = np.empty((len(q), k), dtype=np.float32)
        self._L().hnsw_search(self.h, q.ctypes.data, len(q), self.dim, k, ef, threads, lab.ctypes.data, d.ctypes.data)
        return lab, d

    def free(self):
        if self.h:
            self._L().hnsw_free(self.h)
            self.h = None
