"""Graph containers and the reference's index file formats.

The adjacency layout used everywhere (host and HBM) is the reference's FPGA
link layout: one row per node of 16*(1+ceil(max_degree/16)) int32 words, the
neighbour count in word 0 of a 64-byte header line and the ids from word 16
(vector_search_baselines/scripts_hnsw/hnsw.py:276-297,
scripts_nsg/nsg_to_FPGA.py:81-98).  The kernels read it in place, so the
reference's own index files load without conversion.
"""
import os

import numpy as np


def pad16(d):
    return (d + 15) // 16 * 16


def link_stride(max_degree):
    return 16 * (1 + (max_degree + 15) // 16)


class Graph:
    """A proximity graph over `vectors` with the reference link layout."""

    def __init__(self, vectors, links, max_degree, entry_point, labels=None, ids_offset=16):
        self.vectors = np.ascontiguousarray(vectors, dtype=np.float32)
        self.links = np.ascontiguousarray(links, dtype=np.int32)
        self.max_degree = int(max_degree)
        self.entry_point = int(entry_point)
        self.labels = None if labels is None else np.ascontiguousarray(labels, dtype=np.int32)
        self.ids_offset = int(ids_offset)
        assert self.links.ndim == 2 and self.links.shape[0] == self.vectors.shape[0]

    @property
    def n(self):
        return self.vectors.shape[0]

    @property
    def dim(self):
        return self.vectors.shape[1]

    @classmethod
    def from_adjacency(cls, vectors, adj, entry_point, labels=None):
        """adj: [n, max_degree] int32, -1 after each row's neighbours."""
        adj = np.asarray(adj, dtype=np.int32)
        n, md = adj.shape
        valid = adj >= 0
        counts = valid.sum(axis=1).astype(np.int32)
        # neighbours must be a prefix of the row
        if not np.all(valid == (np.arange(md)[None, :] < counts[:, None])):
            raise ValueError("adjacency rows must hold their neighbours first, then -1")
        rows = np.zeros((n, link_stride(md)), dtype=np.int32)
        rows[:, 0] = counts
        rows[:, 16:16 + md] = np.where(valid, adj, 0)
        return cls(vectors, rows, md, entry_point, labels)

    def counts(self):
        return self.links[:, 0].copy()

    def adjacency(self):
        """[n, max_degree] int32 neighbour ids, -1 padded."""
        md = self.max_degree
        ids = self.links[:, self.ids_offset:self.ids_offset + md].copy()
        ids[np.arange(md)[None, :] >= self.links[:, :1]] = -1
        return ids


# ---------------------------------------------------------------------------
# Reference FPGA index files (hnsw.py:264-377 / nsg_to_FPGA.py:56-137)
# ---------------------------------------------------------------------------

def write_fpga_index(out_dir, graph, graph_type="HNSW", max_level=0, max_m=None, upper=None, num_channels=(1,)):
    """Write meta.bin, ground_links_{nc}_chan_{i}.bin, ground_vectors_{nc}_chan_{i}.bin
    for every nc in num_channels (rows round robin: node j to channel j % nc)
    and ground_labels.bin in the reference layout, and with `upper` (HNSW)
    also upper_links.bin and upper_links_pointers.bin."""
    os.makedirs(out_dir, exist_ok=True)
    n, md, dim = graph.n, graph.max_degree, graph.dim
    if upper is not None:
        max_level, max_m = upper.max_level, upper.max_degree
    if graph_type == "HNSW":
        entry = upper.entry if upper is not None else graph.entry_point
        meta = np.array([n, max_level, entry, max_m if max_m else md // 2, md], dtype=np.int32)
    elif graph_type == "NSG":
        meta = np.array([n, graph.entry_point, md], dtype=np.int32)
    else:
        raise ValueError(graph_type)
    meta.tofile(os.path.join(out_dir, "meta.bin"))
    links = np.zeros((n, link_stride(md)), dtype=np.int32)
    links[:, 0] = graph.links[:, 0]
    links[:, 16:16 + md] = graph.links[:, graph.ids_offset:graph.ids_offset + md]
    links[:, 16:16 + md][np.arange(md)[None, :] >= links[:, :1]] = 0
    for nc in num_channels:
        for c in range(nc):
            links[c::nc].tofile(os.path.join(out_dir, "ground_links_%d_chan_%d.bin" % (nc, c)))
    vec = np.zeros((n, pad16(dim) + 16), dtype=np.float32)
    vec[:, :dim] = graph.vectors
    vec[:, pad16(dim)] = np.frombuffer(np.int32(-1).tobytes(), dtype=np.float32)[0]   # visited tag -1
    for nc in num_channels:
        for c in range(nc):
            vec[c::nc].tofile(os.path.join(out_dir, "ground_vectors_%d_chan_%d.bin" % (nc, c)))
    labels = graph.labels if graph.labels is not None else np.arange(n, dtype=np.int32)
    labels.astype(np.int32).tofile(os.path.join(out_dir, "ground_labels.bin"))
    if upper is not None:
        write_fpga_upper(out_dir, upper)


def fpga_channel_sets(index_dir):
    """Channel counts nc with a ground_links_{nc}_chan_0.bin in the directory."""
    return [nc for nc in (1, 2, 4, 8, 16)
            if os.path.exists(os.path.join(index_dir, "ground_links_%d_chan_0.bin" % nc))]


def read_fpga_index(index_dir, graph_type, dim, channels=None):
    """Read the reference's FPGA files into a Graph.  The writers spread the
    rows round robin over nc channel files, node i as row i // nc of channel
    i % nc (hnsw.py:324-335, nsg_to_FPGA.py:124-135); the rows are put back in
    node order.  channels: the set to read (default: 1 if present, else the
    smallest available)."""
    meta = np.fromfile(os.path.join(index_dir, "meta.bin"), dtype=np.int32)
    if graph_type == "HNSW":
        n, entry, md = int(meta[0]), int(meta[2]), int(meta[4])
    else:
        n, entry, md = int(meta[0]), int(meta[1]), int(meta[2])
    sets = fpga_channel_sets(index_dir)
    nc = channels or (sets[0] if sets else 1)
    links = np.empty((n, link_stride(md)), dtype=np.int32)
    vec = np.empty((n, pad16(dim) + 16), dtype=np.float32)
    for c in range(nc):
        rows = (n - c + nc - 1) // nc
        links[c::nc] = np.fromfile(os.path.join(index_dir, "ground_links_%d_chan_%d.bin" % (nc, c)),
                                   dtype=np.int32).reshape(rows, link_stride(md))
        vec[c::nc] = np.fromfile(os.path.join(index_dir, "ground_vectors_%d_chan_%d.bin" % (nc, c)),
                                 dtype=np.float32).reshape(rows, pad16(dim) + 16)
    lp = os.path.join(index_dir, "ground_labels.bin")
    labels = np.fromfile(lp, dtype=np.int32) if (graph_type == "HNSW" and os.path.exists(lp)) else None
    return Graph(vec[:, :dim], links, md, entry, labels)


def reference_vector_rows(vectors):
    """Vectors in the reference FPGA row layout: pad16(dim) floats + 64-byte pad."""
    n, dim = vectors.shape
    out = np.zeros((n, pad16(dim) + 16), dtype=np.float32)
    out[:, :dim] = vectors
    out[:, pad16(dim)] = np.frombuffer(np.int32(-1).tobytes(), dtype=np.float32)[0]
    return out


# ---------------------------------------------------------------------------
# HNSW upper layers
# ---------------------------------------------------------------------------

class UpperLayers:
    """HNSW levels >= 1 in hnswlib's arrangement: node v is on levels
    0..levels[v]; for 1 <= l <= levels[v] its level-l list is row
    row_start[v] + l - 1 of `rows` ([num_rows, 1 + max_degree] int32: the
    count, then the ids; hnswalg.h:379-381, size_links_per_element_)."""

    def __init__(self, max_level, max_degree, entry, levels, row_start, rows):
        self.max_level = int(max_level)
        self.max_degree = int(max_degree)
        self.entry = int(entry)
        self.levels = np.ascontiguousarray(levels, dtype=np.int32)
        self.row_start = np.ascontiguousarray(row_start, dtype=np.int64)
        self.rows = np.ascontiguousarray(rows, dtype=np.int32).reshape(-1, 1 + self.max_degree)

    def row(self, v, level):
        """Neighbour ids of node v on `level` (>= 1)."""
        r = self.rows[self.row_start[v] + level - 1]
        return r[1:1 + r[0]].copy()

    @classmethod
    def from_lists(cls, max_degree, entry, lists):
        """lists[v] = [ids on level 1, ids on level 2, ...] (empty for base-only nodes)."""
        n = len(lists)
        levels = np.array([len(x) for x in lists], dtype=np.int32)
        row_start = np.zeros(n, dtype=np.int64)
        row_start[1:] = np.cumsum(levels)[:-1]
        rows = np.zeros((max(int(levels.sum()), 1), 1 + max_degree), dtype=np.int32)
        for v, per_level in enumerate(lists):
            for l, ids in enumerate(per_level):
                r = rows[row_start[v] + l]
                r[0] = len(ids)
                r[1:1 + len(ids)] = ids
        return cls(int(levels.max()) if n else 0, max_degree, entry, levels, row_start, rows)


# hnswlib save files (hnswalg.h:588-616 of the reference's vendored hnswlib;
# hnsw.py:139-262 reads the same layout): a 96-byte header, then per element
# (in internal-id order) the level-0 record [count u32 (low 16 bits), maxM0 ids
# u32, dim floats, label u64], then per element [bytes u32, levels x (count u32,
# maxM ids u32)].
_HNSW_HEADER = np.dtype([("offsetLevel0", "<u8"), ("max_elements", "<u8"), ("cur_element_count", "<u8"),
                         ("size_data_per_element", "<u8"), ("label_offset", "<u8"), ("offsetData", "<u8"),
                         ("maxlevel", "<i4"), ("enterpoint_node", "<u4"), ("maxM", "<u8"), ("maxM0", "<u8"),
                         ("M", "<u8"), ("mult", "<f8"), ("ef_construction", "<u8")])


def read_hnswlib_index(path):
    """Read an hnswlib save file.  Returns (Graph of the base layer with the
    file's labels, UpperLayers or None when the index has one level, header
    dict)."""
    raw = np.fromfile(path, dtype=np.uint8)
    hdr = np.frombuffer(raw[:_HNSW_HEADER.itemsize].tobytes(), dtype=_HNSW_HEADER)[0]
    n = int(hdr["cur_element_count"])
    size = int(hdr["size_data_per_element"])
    m0, m = int(hdr["maxM0"]), int(hdr["maxM"])
    off_data, off_label = int(hdr["offsetData"]), int(hdr["label_offset"])
    if int(hdr["offsetLevel0"]) != 0 or off_data != 4 + 4 * m0:
        raise ValueError("unsupported hnswlib layout (offsetLevel0=%d, offsetData=%d)" % (hdr["offsetLevel0"], off_data))
    dim = (off_label - off_data) // 4
    pos = _HNSW_HEADER.itemsize
    rec = raw[pos:pos + n * size].reshape(n, size)
    pos += n * size
    counts = rec[:, 0:4].copy().view("<u4")[:, 0] & 0xffff
    ids = rec[:, 4:off_data].copy().view("<u4").astype(np.int64)
    vectors = rec[:, off_data:off_label].copy().view("<f4")
    labels = rec[:, off_label:off_label + 8].copy().view("<u8")[:, 0]
    adj = np.where(np.arange(m0)[None, :] < counts[:, None], ids, -1).astype(np.int32)
    levels = np.zeros(n, dtype=np.int32)
    row_start = np.zeros(n, dtype=np.int64)
    chunks = []
    row_bytes = 4 * (1 + m)
    nrows = 0
    for v in range(n):
        nb = int(np.frombuffer(raw[pos:pos + 4].tobytes(), dtype="<u4")[0])
        pos += 4
        row_start[v] = nrows
        if nb:
            lv = nb // row_bytes
            levels[v] = lv
            block = raw[pos:pos + nb].copy().view("<u4").reshape(lv, 1 + m).astype(np.int64)
            block[:, 0] &= 0xffff
            # slots past the count may hold stale ids: clear them
            block[:, 1:][np.arange(m)[None, :] >= block[:, :1]] = 0
            chunks.append(block.astype(np.int32))
            nrows += lv
            pos += nb
    if pos != raw.size:
        raise ValueError("trailing bytes in %s" % path)
    entry = int(hdr["enterpoint_node"])
    g = Graph.from_adjacency(vectors, adj, entry, labels=labels.astype(np.int32))
    upper = None
    if int(hdr["maxlevel"]) > 0:
        rows = np.concatenate(chunks) if chunks else np.zeros((1, 1 + m), dtype=np.int32)
        upper = UpperLayers(int(hdr["maxlevel"]), m, entry, levels, row_start, rows)
    info = {k: (float(hdr[k]) if k == "mult" else int(hdr[k])) for k in _HNSW_HEADER.names}
    info["dim"] = dim
    return g, upper, info


def write_hnswlib_index(path, graph, upper, M, ef_construction=200, labels=None):
    """Write `graph` (base layer, max_degree = maxM0) and `upper` (or None) as
    an hnswlib save file that hnswlib's loadIndex reads."""
    n, dim, m0 = graph.n, graph.dim, graph.max_degree
    m = upper.max_degree if upper is not None else M
    size = 4 + 4 * m0 + 4 * dim + 8
    hdr = np.zeros(1, dtype=_HNSW_HEADER)
    hdr["offsetLevel0"], hdr["max_elements"], hdr["cur_element_count"] = 0, n, n
    hdr["size_data_per_element"], hdr["label_offset"], hdr["offsetData"] = size, 4 + 4 * m0 + 4 * dim, 4 + 4 * m0
    hdr["maxlevel"] = upper.max_level if upper is not None else 0
    hdr["enterpoint_node"] = upper.entry if upper is not None else graph.entry_point
    hdr["maxM"], hdr["maxM0"], hdr["M"] = m, m0, M
    hdr["mult"] = 1.0 / np.log(float(M))
    hdr["ef_construction"] = ef_construction
    rec = np.zeros((n, size), dtype=np.uint8)
    adj = graph.adjacency()
    rec[:, 0:4] = graph.counts().astype("<u4").view(np.uint8).reshape(n, 4)
    rec[:, 4:4 + 4 * m0] = np.where(adj >= 0, adj, 0).astype("<u4").view(np.uint8).reshape(n, 4 * m0)
    rec[:, 4 + 4 * m0:4 + 4 * m0 + 4 * dim] = graph.vectors.astype("<f4").view(np.uint8).reshape(n, 4 * dim)
    lab = labels if labels is not None else (graph.labels if graph.labels is not None else np.arange(n))
    rec[:, size - 8:] = np.asarray(lab, dtype="<u8").view(np.uint8).reshape(n, 8)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(rec.tobytes())
        for v in range(n):
            lv = int(upper.levels[v]) if upper is not None else 0
            f.write(np.uint32(lv * 4 * (1 + m)).tobytes())
            if lv:
                f.write(upper.rows[upper.row_start[v]:upper.row_start[v] + lv].astype("<u4").tobytes())


# Reference multi-layer FPGA files (hnsw.py:264-377; read by FPGA_single_DDR/
# FPGA_single_DDR_multi_layer_v2.2_async/src/host.cpp:66-161): upper_links.bin
# holds, per node and level, a 64-byte header line (count + 60 bytes of zeros)
# and then maxM ids padded to 64 bytes; upper_links_pointers.bin holds one
# 8-byte byte offset per node.

def _fpga_upper_row_words(max_m):
    return 16 * (1 + (4 * max_m + 63) // 64)


def write_fpga_upper(out_dir, upper):
    n = upper.levels.shape[0]
    rw = _fpga_upper_row_words(upper.max_degree)
    ptr = np.zeros(n, dtype="<u8")
    blocks = []
    off = 0
    for v in range(n):
        ptr[v] = off
        for l in range(1, int(upper.levels[v]) + 1):
            r = upper.rows[upper.row_start[v] + l - 1]
            row = np.zeros(rw, dtype="<u4")
            row[0] = r[0]
            row[16:16 + upper.max_degree] = np.where(np.arange(upper.max_degree) < r[0], r[1:], 0)
            blocks.append(row)
            off += 4 * rw
    data = np.concatenate(blocks) if blocks else np.zeros(0, dtype="<u4")
    data.tofile(os.path.join(out_dir, "upper_links.bin"))
    ptr.tofile(os.path.join(out_dir, "upper_links_pointers.bin"))


def read_fpga_upper(index_dir):
    """UpperLayers from meta.bin (n, max_level, entry, maxM, maxM0) and the
    upper-link files, or None when max_level is 0 or the files are absent."""
    meta = np.fromfile(os.path.join(index_dir, "meta.bin"), dtype=np.int32)
    n, max_level, entry, max_m = int(meta[0]), int(meta[1]), int(meta[2]), int(meta[3])
    lp, pp = os.path.join(index_dir, "upper_links.bin"), os.path.join(index_dir, "upper_links_pointers.bin")
    if max_level < 1 or not (os.path.exists(lp) and os.path.exists(pp)):
        return None
    rw = _fpga_upper_row_words(max_m)
    data = np.fromfile(lp, dtype="<u4").reshape(-1, rw).astype(np.int64)
    ptr = np.fromfile(pp, dtype="<u8").astype(np.int64)
    if ptr.shape[0] != n:
        raise ValueError("upper_links_pointers.bin holds %d pointers for %d nodes" % (ptr.shape[0], n))
    ends = np.append(ptr[1:], data.shape[0] * 4 * rw)
    levels = ((ends - ptr) // (4 * rw)).astype(np.int32)
    row_start = (ptr // (4 * rw)).astype(np.int64)
    rows = np.zeros((max(data.shape[0], 1), 1 + max_m), dtype=np.int32)
    if data.shape[0]:
        rows[:data.shape[0], 0] = data[:, 0]
        rows[:data.shape[0], 1:] = data[:, 16:16 + max_m]
    return UpperLayers(max_level, max_m, entry, levels, row_start, rows)


# ---------------------------------------------------------------------------
# NSG graph files and dataset vector files read by the reference's scripts
# ---------------------------------------------------------------------------

def read_nsg_index(path, vectors):
    """An NSG save file (the format nsg_to_FPGA.py:31-47 reads: width u32,
    entry point u32, then per node a count u32 and that many ids u32) over
    `vectors` as a Graph; max degree = the file's width (or the longest row)."""
    raw = np.fromfile(path, dtype="<u4")
    width, ep = int(raw[0]), int(raw[1])
    n = vectors.shape[0]
    rows, pos = [], 2
    while pos < raw.size:
        k = int(raw[pos])
        rows.append(raw[pos + 1:pos + 1 + k].astype(np.int64))
        pos += 1 + k
    if len(rows) != n:
        raise ValueError("%s holds %d rows for %d vectors" % (path, len(rows), n))
    md = max(width, max((len(r) for r in rows), default=0))
    adj = np.full((n, md), -1, dtype=np.int32)
    for i, r in enumerate(rows):
        adj[i, :len(r)] = r
    return Graph.from_adjacency(vectors, adj, ep)


def write_nsg_index(path, graph):
    """Write `graph` as an NSG save file (width = max degree)."""
    adj = graph.adjacency()
    out = [np.array([graph.max_degree, graph.entry_point], dtype="<u4")]
    for row in adj:
        r = row[row >= 0]
        out.append(np.array([len(r)], dtype="<u4"))
        out.append(r.astype("<u4"))
    np.concatenate(out).tofile(path)


def read_fvecs(path):
    """TEXMEX .fvecs: per row an int32 dimension, then that many float32."""
    a = np.fromfile(path, dtype="<i4")
    d = int(a[0])
    return a.reshape(-1, d + 1)[:, 1:].view("<f4").copy()


def read_ivecs(path):
    """TEXMEX .ivecs (ground-truth ids): per row an int32 count, then int32 ids."""
    a = np.fromfile(path, dtype="<i4")
    d = int(a[0])
    return a.reshape(-1, d + 1)[:, 1:].copy()


def read_bvecs(path):
    """TEXMEX .bvecs (SIFT1B): per row an int32 dimension, then uint8 values; as float32."""
    a = np.fromfile(path, dtype=np.uint8)
    d = int(a[:4].view("<i4")[0])
    return a.reshape(-1, d + 4)[:, 4:].astype(np.float32)


def read_bin(path, dtype="<f4"):
    """big-ann-benchmarks .fbin / .ibin / .u8bin: n u32, dim u32, then n x dim values."""
    n, d = (int(v) for v in np.fromfile(path, dtype="<u4", count=2))
    return np.fromfile(path, dtype=dtype, offset=8).reshape(n, d)


def write_vecs(path, array):
    """Write a TEXMEX .fvecs (float32), .ivecs (int32) or .bvecs (uint8) file by the array's dtype."""
    a = np.ascontiguousarray(array)
    n, d = a.shape
    with open(path, "wb") as f:
        for row in a:
            f.write(np.int32(d).tobytes())
            f.write(row.tobytes())
