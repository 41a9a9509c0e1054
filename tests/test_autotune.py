"""Autotuner: Bloom sizing from visited counts (CPU), profile storage and
lookup (CPU), and one small measured tune on the GPU."""
import math

import numpy as np
import pytest

from helpers import small_graph


def test_bloom_bits_for_false_rejection_target():
    from falcon_b200.autotune import bloom_bits_for
    prev = 0
    for v in (100, 2000, 20000, 60000, 500000):
        b = bloom_bits_for(v, 0.01)
        assert b >= prev
        prev = b
        if b < 24:
            assert (1 - math.exp(-3 * v / (1 << b))) ** 3 <= 0.01
        if b > 16:
            assert (1 - math.exp(-3 * v / (1 << (b - 1)))) ** 3 > 0.01
    assert bloom_bits_for(2000, 0.01) == 16      # the reference's 2^16 suffices at ef=64 on SIFT-like visits


def test_profile_roundtrip_and_pick(tmp_path):
    from falcon_b200.autotune import load_profile, pick, save_profile, best_for_recall
    prof = {
        "D96_R64_ef64": {"throughput": {"params": {"k": 10, "ef": 64, "mc": 1, "mg": 1, "cand_queue_size": 32,
                                                   "bloom_bits": 16, "mode": "inter"}, "qps": 1.5e6, "recall": 0.3},
                         "latency": {"threads_per_query": 32, "mode": "inter", "channels": None, "median_ms": {}}},
        "D96_R64_ef1024": {"throughput": {"params": {"k": 10, "ef": 1024, "mc": 1, "mg": 1, "cand_queue_size": 256,
                                                     "bloom_bits": 20, "mode": "inter"}, "qps": 7e4, "recall": 0.96},
                           "latency": {"threads_per_query": 416, "mode": "intra", "channels": 8, "mc": 2, "mg": 4,
                                       "bloom_bits": 18, "median_ms": {}}},
    }
    path = str(tmp_path / "p.json")
    save_profile(prof, path)
    got = load_profile(path)
    assert pick(got, 96, 64, 500)["ef"] == 1024
    lp = pick(got, 96, 64, 1024, objective="latency")
    assert (lp["channels"], lp["mc"], lp["mg"], lp["bloom_bits"]) == (8, 2, 4, 18)     # DST setting of the latency pick
    assert pick(got, 96, 64, 1024)["mg"] == 1                                          # throughput keeps its own
    assert best_for_recall(got, 0.95)[0] == "D96_R64_ef1024"
    with pytest.raises(KeyError):
        pick(got, 128, 64, 64)


@pytest.mark.gpu
def test_tune_small_index():
    from falcon_b200 import FalconIndex
    from falcon_b200.autotune import tune
    from falcon_b200.groundtruth import brute_force_f64
    g, q = small_graph("unit", 6000, 96, 64, 200, seed=41)
    ix = FalconIndex(g)
    gt, _ = brute_force_f64(g.vectors, q, 10)
    prof = tune(ix, q, gt, 96, 64, ef_list=(32, 128), recall_target=0.9, cq_grid=(32, 64),
                mcmg_grid=((1, 1), (2, 2)), latency_channels=(4,))
    assert set(prof) == {"D96_R64_ef32", "D96_R64_ef128"}
    for e in prof.values():
        t = e["throughput"]
        assert t["qps"] > 0 and 0 <= t["recall"] <= 1
        if e["recall_target_met"]:
            assert t["recall"] >= 0.9
        lat = e["latency"]
        assert lat["mode"] in ("inter", "intra") and lat["mc"] >= 1 and lat["mg"] >= 1
        # a latency setting may not cost recall beyond the tolerance (or below a met target)
        need = min(0.9, t["recall"] - 0.002) if e["recall_target_met"] else t["recall"] - 0.002
        assert lat["recall"] >= need - 1e-9
    assert prof["D96_R64_ef128"]["throughput"]["recall"] >= prof["D96_R64_ef32"]["throughput"]["recall"]
    # the server takes a request's parameters from the profile
    from falcon_b200.serving import FalconServer
    sv = FalconServer(ring_capacity=256, max_k=10, ef_max=128, cand_queue_max=64, dim_max=96, idle_exit_us=2000)
    iid = sv.add_index(ix)
    sv.set_profile(prof)
    p = sv.auto_params(iid, k=10, ef=100)
    want = prof["D96_R64_ef128"]["throughput"]["params"]     # the entry at or above the requested ef
    assert (p.ef, p.mc, p.mg, p.cand_queue_size, p.bloom_bits) == (100, want["mc"], want["mg"],
                                                                    want["cand_queue_size"], want["bloom_bits"])
    rid = sv.submit([iid], q[:1], p)
    ids, d, hops, vis = sv.wait(rid[0], 10)
    r = ix.search(q[:1], k=10, ef=p.ef, mc=p.mc, mg=p.mg, cand_queue_size=p.cand_queue_size, bloom_bits=p.bloom_bits)
    assert np.array_equal(ids, r.ids[0]) and hops == r.hops[0]
    sv.close()


def test_channel_bloom_bits():
    """Each intra-query channel sees 1/channels of the ids: a filter of
    bits - log2(channels) + 1 has at most the whole-query false-rejection rate;
    shared-memory filters stop at 2^18 bits."""
    import math
    from falcon_b200.autotune import channel_bloom_bits
    assert channel_bloom_bits(19, 4) == 18 and channel_bloom_bits(19, 8) == 17 and channel_bloom_bits(22, 2) == 18
    assert channel_bloom_bits(16, 1) == 17 - 0 - 0 and channel_bloom_bits(10, 8) == 10
    for bits in range(14, 21):
        for ch in (2, 4, 8):
            v = 0.3 * (1 << bits) / 3        # visited ids filling ~26 % of the whole-query filter
            whole = (1 - math.exp(-3 * v / (1 << bits))) ** 3
            b = channel_bloom_bits(bits, ch)
            if b < 18:
                per = (1 - math.exp(-3 * (v / ch) / (1 << b))) ** 3
                assert per <= whole
