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

def write_fpga_index(out_dir, graph, graph_type="HNSW", max_level=0, max_m=None):
    """Write meta.bin, ground_links_1_chan_0.bin, ground_vectors_1_chan_0.bin
    and ground_labels.bin in the reference layout (single channel)."""
    os.makedirs(out_dir, exist_ok=True)
    n, md, dim = graph.n, graph.max_degree, graph.dim
    if graph_type == "HNSW":
        meta = np.array([n, max_level, graph.entry_point, max_m if max_m else md // 2, md], dtype=np.int32)
    elif graph_type == "NSG":
        meta = np.array([n, graph.entry_point, md], dtype=np.int32)
    else:
        raise ValueError(graph_type)
    meta.tofile(os.path.join(out_dir, "meta.bin"))
    links = np.zeros((n, link_stride(md)), dtype=np.int32)
    links[:, 0] = graph.links[:, 0]
    links[:, 16:16 + md] = graph.links[:, graph.ids_offset:graph.ids_offset + md]
    links[:, 16:16 + md][np.arange(md)[None, :] >= links[:, :1]] = 0
    links.tofile(os.path.join(out_dir, "ground_links_1_chan_0.bin"))
    vec = np.zeros((n, pad16(dim) + 16), dtype=np.float32)
    vec[:, :dim] = graph.vectors
    vec[:, pad16(dim)] = np.frombuffer(np.int32(-1).tobytes(), dtype=np.float32)[0]   # visited tag -1
    vec.tofile(os.path.join(out_dir, "ground_vectors_1_chan_0.bin"))
    labels = graph.labels if graph.labels is not None else np.arange(n, dtype=np.int32)
    labels.astype(np.int32).tofile(os.path.join(out_dir, "ground_labels.bin"))


def read_fpga_index(index_dir, graph_type, dim):
    """Read the reference's single-channel FPGA files into a Graph."""
    meta = np.fromfile(os.path.join(index_dir, "meta.bin"), dtype=np.int32)
    if graph_type == "HNSW":
        n, entry, md = int(meta[0]), int(meta[2]), int(meta[4])
    else:
        n, entry, md = int(meta[0]), int(meta[1]), int(meta[2])
    links = np.fromfile(os.path.join(index_dir, "ground_links_1_chan_0.bin"), dtype=np.int32).reshape(n, link_stride(md))
    vec = np.fromfile(os.path.join(index_dir, "ground_vectors_1_chan_0.bin"), dtype=np.float32).reshape(n, pad16(dim) + 16)
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
