"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

Needs the reference checkout (only in the build container), because every
expected value comes from the reference's own code:
  murmur2_keylen4.json   unit_tests/bloom_and_hash/sw_murmur2/murmur2.cpp
                         (MurmurHash2 and MurmurHash2_KeyLen4), via
                         oracle/_ref/murmur_golden
  bloom_sw_stream.npz    unit_tests/bloom_and_hash/sw_bloom/bloom_murmur2.hpp
                         BloomFilter::check_and_insert, via oracle/_ref/bloom_golden
  traversal_*.npz        the inter-query v1.3 HLS kernel pipeline run as C++
                         (oracle/_ref/libfalcon_ref_d{D}.so) on a seeded graph:
                         ids, distances, hops and visited per query and
                         parameter set.
  intra_v15_d96_md64.npz the intra-query v1.5 HLS kernel pipeline run as C++
                         (oracle/_ref/libfalcon_ref_intra_d96_c{2,4}.so, the
                         nodes spread round robin over 2 or 4 channels) on a
                         seeded unit-normal graph (no repeated distances, so the
                         readiness-order channel merge is schedule independent):
                         ids, distances and hops per query and parameter set.
The graph is stored in the fixture (int16 adjacency); vectors and queries are
regenerated from their seeds (integer-valued for the traversal fixtures), so
the fixtures stay small.

usage: python tests/golden/make_golden.py
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "falcon-accelerate-graph-vector-search_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import build_oracle  # noqa: E402
import oracle  # noqa: E402
from falcon_b200.graph import build_graph  # noqa: E402
from falcon_b200.synthetic import sift_like, unit_normal  # noqa: E402

TRAVERSAL_CASES = [
    # name, n, dim, max_degree, n_queries, parameter sets (ef, mc, mg, cand_queue_size, bloom_bits)
    ("traversal_d128_md32", 1500, 128, 32, 16,
     [(64, 1, 1, 32, 16), (64, 1, 4, 32, 16), (32, 2, 3, 32, 16), (16, 4, 2, 16, 12), (128, 2, 6, 32, 16)]),
    ("traversal_d96_md64", 1500, 96, 64, 16,
     [(64, 1, 1, 32, 16), (64, 2, 5, 32, 16), (48, 1, 2, 24, 14)]),
]

INTRA_CASE = ("intra_v15_d96_md64", 1500, 96, 64, 16,
              # channels, ef, mc, mg, bloom_bits
              [(2, 64, 1, 1, 15), (4, 64, 2, 6, 14), (4, 128, 4, 3, 15), (2, 32, 2, 2, 16)])


def main():
    if not build_oracle.build_ref():
        sys.exit("reference checkout not found; fixtures need the reference's own code")
    out = subprocess.run([os.path.join(build_oracle.REF_OUT, "murmur_golden")], check=True,
                         stdout=subprocess.PIPE, text=True).stdout
    json.dump(json.loads(out), open(os.path.join(HERE, "murmur2_keylen4.json"), "w"), indent=0)
    out = subprocess.run([os.path.join(build_oracle.REF_OUT, "bloom_golden"), "16", "20000"], check=True,
                         stdout=subprocess.PIPE, text=True).stdout
    bl = json.loads(out)
    np.savez_compressed(os.path.join(HERE, "bloom_sw_stream.npz"), bits=np.int32(bl["bits"]), seed=np.int32(bl["seed"]),
                        keys=np.array(bl["keys"], dtype=np.int32), valid=np.array(bl["valid"], dtype=np.uint8))
    for name, n, dim, md, nq, psets in TRAVERSAL_CASES:
        x = sift_like(n, dim, seed=11)
        q = sift_like(nq, dim, seed=12)
        g = build_graph(x, md, device="cpu")
        adj = g.adjacency()
        assert adj.max() < 32768
        res = {}
        for i, (ef, mc, mg, cq, bits) in enumerate(psets):
            ids, d, hops, vis = oracle.ref_inter_search(g.vectors, g.links, md, q, g.entry_point, ef=ef,
                                                        cand_queue_size=cq, mc=mc, mg=mg, bloom_bits=bits)
            res["ids_%d" % i], res["dists_%d" % i], res["hops_%d" % i], res["visited_%d" % i] = ids, d, hops, vis
        np.savez_compressed(os.path.join(HERE, name + ".npz"), adjacency=adj.astype(np.int16),
                            entry=np.int32(g.entry_point), data_seed=np.int32(11), query_seed=np.int32(12),
                            n=np.int32(n), dim=np.int32(dim), max_degree=np.int32(md), n_queries=np.int32(nq),
                            params=np.array(psets, dtype=np.int32), **res)
        print(name, "written")
    name, n, dim, md, nq, psets = INTRA_CASE
    x = unit_normal(n, dim, seed=13)
    q = unit_normal(nq, dim, seed=14)
    g = build_graph(x, md, device="cpu")
    adj = g.adjacency()
    res = {}
    for i, (ch, ef, mc, mg, bits) in enumerate(psets):
        ids, d, hops = oracle.ref_intra_search(g.vectors, g.links, md, q, g.entry_point, ch, ef=ef, mc=mc, mg=mg,
                                               bloom_bits=bits)
        res["ids_%d" % i], res["dists_%d" % i], res["hops_%d" % i] = ids, d, hops
    np.savez_compressed(os.path.join(HERE, name + ".npz"), adjacency=adj.astype(np.int16),
                        entry=np.int32(g.entry_point), data_seed=np.int32(13), query_seed=np.int32(14),
                        n=np.int32(n), dim=np.int32(dim), max_degree=np.int32(md), n_queries=np.int32(nq),
                        params=np.array(psets, dtype=np.int32), **res)
    print(name, "written")


if __name__ == "__main__":
    main()
