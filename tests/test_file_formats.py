"""CPU: the graph and dataset files the reference's scripts read — NSG save
files (nsg_to_FPGA.py:31-47) and the TEXMEX / big-ann vector files
(scripts_nsg/utils.py: mmap_fvecs, mmap_bvecs, ivecs_read, read_deep_fbin)."""
import numpy as np

from helpers import small_graph


def test_nsg_round_trip(tmp_path):
    from falcon_b200.formats import read_nsg_index, write_nsg_index
    g, _ = small_graph("sift", 2000, 128, 32, 4, seed=3)
    p = str(tmp_path / "g.nsg")
    write_nsg_index(p, g)
    raw = np.fromfile(p, dtype="<u4")
    assert raw[0] == 32 and raw[1] == g.entry_point and raw[2] == g.counts()[0]
    assert raw.size == 2 + g.n + int(g.counts().sum())
    g2 = read_nsg_index(p, g.vectors)
    assert np.array_equal(g2.adjacency(), g.adjacency()) and g2.entry_point == g.entry_point
    assert np.array_equal(g2.links, g.links)


def test_nsg_rows_longer_than_width(tmp_path):
    from falcon_b200.formats import read_nsg_index
    x = np.zeros((3, 16), dtype=np.float32)
    rows = [[1, 2], [0, 2, 1], [0]]
    data = [2, 1] + sum(([len(r)] + r for r in rows), [])
    p = str(tmp_path / "h.nsg")
    np.array(data, dtype="<u4").tofile(p)
    g = read_nsg_index(p, x)
    assert g.max_degree == 3 and g.entry_point == 1
    assert g.adjacency().tolist() == [[1, 2, -1], [0, 2, 1], [0, -1, -1]]


def test_texmex_and_bin_files(tmp_path):
    from falcon_b200.formats import read_bin, read_bvecs, read_fvecs, read_ivecs, write_vecs
    rng = np.random.default_rng(0)
    f = rng.standard_normal((7, 96)).astype(np.float32)
    i = rng.integers(0, 1000, (7, 100)).astype(np.int32)
    b = rng.integers(0, 256, (7, 128)).astype(np.uint8)
    write_vecs(str(tmp_path / "a.fvecs"), f)
    write_vecs(str(tmp_path / "a.ivecs"), i)
    write_vecs(str(tmp_path / "a.bvecs"), b)
    assert np.array_equal(read_fvecs(str(tmp_path / "a.fvecs")), f)
    assert np.array_equal(read_ivecs(str(tmp_path / "a.ivecs")), i)
    assert np.array_equal(read_bvecs(str(tmp_path / "a.bvecs")), b.astype(np.float32))
    with open(str(tmp_path / "a.fbin"), "wb") as fh:
        fh.write(np.array([7, 96], dtype="<u4").tobytes())
        fh.write(f.tobytes())
    assert np.array_equal(read_bin(str(tmp_path / "a.fbin")), f)
