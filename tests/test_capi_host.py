"""CPU: the C-ABI library loads and exports every declared symbol; host-side
logic (file formats, graph builder, ground truth, recall) behaves."""
import os
import re

import numpy as np
import pytest

from helpers import small_graph

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(REPO, "include", "falcon.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(falcon_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lib):
    from falcon_b200 import _lib
    names = declared_functions()
    assert len(names) >= 9
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, n


def test_build_info_and_defaults(lib):
    from falcon_b200 import _lib
    assert b"sm_100a" in lib.falcon_build_info()
    p = _lib.SearchParams()
    lib.falcon_default_params(p)
    assert (p.k, p.ef, p.mc, p.mg, p.cand_queue_size, p.bloom_bits, p.hash_seed) == (10, 64, 1, 1, 32, 16, 1)


def test_struct_layouts_match_header(tmp_path):
    """Every struct the ctypes binding mirrors has the header's size and field
    offsets (compiled with the system C compiler)."""
    import ctypes
    import subprocess
    from falcon_b200 import _lib
    assert ctypes.sizeof(_lib.IndexDesc) == 72
    assert ctypes.sizeof(_lib.SearchParams) == 48
    assert ctypes.sizeof(_lib.IndexInfo) == 40
    pairs = [("falcon_index_desc", _lib.IndexDesc), ("falcon_index_info", _lib.IndexInfo),
             ("falcon_search_params", _lib.SearchParams), ("falcon_upper_layers_desc", _lib.UpperLayersDesc),
             ("falcon_server_config", _lib.ServerConfig), ("falcon_server_info", _lib.ServerInfo)]
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "falcon.h"', "int main(void) {"]
    for cname, cls in pairs:
        lines.append('printf("%%zu\\n", sizeof(%s));' % cname)
        for f, _ in cls._fields_:
            lines.append('printf("%%zu\\n", offsetof(%s, %s));' % (cname, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", inc, str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = []
    for _, cls in pairs:
        want.append(ctypes.sizeof(cls))
        want += [getattr(cls, f).offset for f, _ in cls._fields_]
    assert got == want


def test_null_arguments_return_errors_without_gpu(lib):
    import ctypes
    from falcon_b200 import _lib
    h = ctypes.c_void_p()
    assert lib.falcon_index_create(None, ctypes.byref(h)) == _lib.FALCON_ERR_ARG
    assert b"null" in lib.falcon_last_error()
    assert lib.falcon_search(None, None, 0, 0, None, None, 0, None, None, 0, None, None, 0, None) == _lib.FALCON_ERR_ARG
    assert lib.falcon_index_free(None) == _lib.FALCON_OK


def test_graph_validation_rejects_bad_rows(lib):
    """Malformed graphs are refused on the host before any device work."""
    from falcon_b200 import _lib
    from falcon_b200.formats import Graph
    g, _ = small_graph("sift", 2000, 128, 32, 4, seed=3)
    bad = Graph(g.vectors, g.links.copy(), g.max_degree, g.entry_point)
    bad.links[5, 0] = 33                         # degree > max_degree
    with pytest.raises(_lib.FalconError) as e:
        from falcon_b200 import FalconIndex
        FalconIndex(bad)
    assert e.value.code == _lib.FALCON_ERR_GRAPH
    bad.links[5, 0] = 3
    bad.links[5, 16] = 2000                      # id out of range
    with pytest.raises(_lib.FalconError) as e:
        FalconIndex(bad)
    assert e.value.code == _lib.FALCON_ERR_GRAPH
    bad2 = Graph(g.vectors, g.links, g.max_degree, 5000)   # entry out of range
    with pytest.raises(_lib.FalconError):
        FalconIndex(bad2)


def test_fpga_files_roundtrip(tmp_path):
    from falcon_b200.formats import read_fpga_index, write_fpga_index
    g, _ = small_graph("sift", 2000, 128, 32, 4, seed=3)
    for gt in ("HNSW", "NSG"):
        d = tmp_path / gt
        write_fpga_index(str(d), g, gt)
        r = read_fpga_index(str(d), gt, 128)
        assert np.array_equal(r.vectors, g.vectors)
        assert np.array_equal(r.adjacency(), g.adjacency())
        assert r.entry_point == g.entry_point and r.max_degree == g.max_degree
        # file sizes as the reference host expects (host.cpp:237-278)
        assert os.path.getsize(d / "ground_links_1_chan_0.bin") == 2000 * (64 + 2 * 64)
        assert os.path.getsize(d / "ground_vectors_1_chan_0.bin") == 2000 * (512 + 64)


def test_multichannel_fpga_files(tmp_path):
    """The reference writers' round robin (hnsw.py:324-335, nsg_to_FPGA.py:
    124-135): node j is row j // nc of channel j % nc; reading puts the rows
    back in node order, whichever channel set is present."""
    from falcon_b200.formats import fpga_channel_sets, read_fpga_index, write_fpga_index
    g, _ = small_graph("sift", 1001, 128, 32, 4, seed=5)   # 1001 rows: uneven channels
    d = tmp_path / "mc"
    write_fpga_index(str(d), g, "NSG", num_channels=(2, 4))
    assert fpga_channel_sets(str(d)) == [2, 4]
    row_l, row_v = 64 + 2 * 64, 512 + 64
    for nc in (2, 4):
        for c in range(nc):
            rows = (1001 - c + nc - 1) // nc
            assert os.path.getsize(d / ("ground_links_%d_chan_%d.bin" % (nc, c))) == rows * row_l
            assert os.path.getsize(d / ("ground_vectors_%d_chan_%d.bin" % (nc, c))) == rows * row_v
        # row 3 of channel 1 is node 3 * nc + 1
        raw = np.fromfile(d / ("ground_links_%d_chan_1.bin" % nc), dtype=np.int32).reshape(-1, row_l // 4)
        assert raw[3, 0] == g.counts()[3 * nc + 1]
        assert np.array_equal(raw[3, 16:16 + raw[3, 0]], g.adjacency()[3 * nc + 1, :raw[3, 0]])
        r = read_fpga_index(str(d), "NSG", 128, channels=nc)
        assert np.array_equal(r.vectors, g.vectors) and np.array_equal(r.adjacency(), g.adjacency())
    r = read_fpga_index(str(d), "NSG", 128)
    assert np.array_equal(r.adjacency(), g.adjacency())


def test_graph_builder_properties():
    g, _ = small_graph("unit", 2000, 96, 64, 4, seed=5)
    adj = g.adjacency()
    assert adj.shape == (2000, 64)
    cnt = g.counts()
    assert cnt.min() >= 1 and cnt.max() <= 64
    for r in range(0, 2000, 97):
        row = adj[r, :cnt[r]]
        assert len(set(row.tolist())) == len(row)     # no duplicate edges
        assert r not in row                             # no self loops
        assert np.all(adj[r, cnt[r]:] == -1)


def test_groundtruth_and_recall():
    from falcon_b200.groundtruth import brute_force_f64, recall_at_1, recall_at_k
    rng = np.random.default_rng(0)
    base = rng.standard_normal((3000, 32)).astype(np.float32)
    q = rng.standard_normal((50, 32)).astype(np.float32)
    ids, d = brute_force_f64(base, q, 10)
    full = ((q[:, None, :].astype(np.float64) - base[None].astype(np.float64)) ** 2).sum(-1)
    ref = np.argsort(full, axis=1, kind="stable")[:, :10]
    assert np.array_equal(ids, ref)
    assert np.allclose(d, np.take_along_axis(full, ref, 1))
    assert recall_at_k(ids, ref, 10) == 1.0 and recall_at_1(ids, ref) == 1.0
    shifted = np.concatenate([ids[:, 5:], ids[:, :5] + 100000], 1)
    assert recall_at_k(shifted, ref, 10) == 0.5


def test_synthetic_distributions():
    from falcon_b200.synthetic import sift_like, unit_normal
    s = sift_like(1000, 128, 0)
    assert s.min() >= 0 and s.max() <= 255 and np.all(s == np.rint(s))
    assert np.array_equal(s, sift_like(1000, 128, 0))
    u = unit_normal(1000, 96, 0)
    assert np.allclose(np.linalg.norm(u, axis=1), 1.0, atol=1e-5)
