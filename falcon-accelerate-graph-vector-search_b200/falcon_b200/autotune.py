"""Autotuner: per (dimension, max degree, ef), the traversal configuration.

The reference's only tuner is the networked client's "auto" mode, which takes
mc/mg from the best row of a profiled sweep
(networked_FPGA/CPU_programs/launch_CPU_and_FPGA.py:172-182).  This tuner
measures on the device, for an index and a query sample with ground truth:

  * Bloom size: the smallest filter whose false-rejection rate at the measured
    visited count stays under `fp_target` (a query that visits V nodes sets
    ~3V bits of 2^b; a new node is wrongly rejected with probability
    (1 - exp(-3V/2^b))^3), and the next smaller one: filters above 2^18 bits
    live in global memory, one per resident warp, and halving them can matter
    more for speed (L2 footprint) than the few extra false rejections cost in
    recall, so both are measured;
  * candidate-queue capacity and mc/mg: a grid, keeping the fastest point whose
    recall@k meets the target;
  * threads per query: inter-query (one warp) for throughput; for batch-1
    latency, intra-query blocks of 4 or 8 channels (12 fetch warps and a merge
    warp) are timed as well, each channel with a filter sized for the ids it
    sees (channel_bloom_bits), and at several (mc, mg): the intra kernel
    overlaps a group's fetch with the previous group's merge when mg >= 2.

Profiles are JSON files keyed "D{dim}_R{degree}_ef{ef}".
"""
import json
import math
import os

import numpy as np


def bloom_bits_for(visited, fp_target=0.01, lo=16, hi=24):
    """Smallest b in [lo, hi] with (1 - exp(-3 V / 2^b))^3 <= fp_target."""
    v = max(1.0, float(visited))
    for b in range(lo, hi + 1):
        if (1.0 - math.exp(-3.0 * v / (1 << b))) ** 3 <= fp_target:
            return b
    return hi


def channel_bloom_bits(bits, channels, smem_max=18):
    """Per-channel filter size in intra-query mode: each channel's filter sees
    1/channels of the ids, so bits - log2(channels) + 1 keeps (with a bit to
    spare) the false-rejection rate of a `bits` whole-query filter; capped at
    the largest shared-memory filter, 2^18 bits."""
    return max(10, min(smem_max, bits - int(round(math.log2(channels))) + 1))


def _time_batch(ix, dq, reps=2, **p):
    import torch
    ix.search(dq, **p)
    torch.cuda.synchronize()
    best = float("inf")
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    for _ in range(reps):
        a.record()
        r = ix.search(dq, **p)
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best, r


def _time_single(ix, dq, n=50, **p):
    import torch
    ts = []
    for i in range(n):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        ix.search(dq[i:i + 1], **p)
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts[5:]))


def profile_key(dim, degree, ef):
    return "D%d_R%d_ef%d" % (dim, degree, ef)


def tune(index, queries, gt, dim, degree, ef_list=(64, 128, 256, 512, 1024), k=10, recall_target=0.95,
         fp_target=0.01, cq_grid=(32, 64, 256), mcmg_grid=((1, 1), (2, 1), (1, 4)), latency_channels=(4, 8),
         latency_mcmg=((1, 1), (1, 2), (2, 4)), log=None):
    """Measure and return a profile dict {key: entry}; each entry holds the
    throughput-optimal parameters, their QPS and recall, whether the target was
    met, and the batch-1 latency per threads-per-query choice.  For latency the
    intra-query kernel is also timed at the (mc, mg) of latency_mcmg: with mg >=
    2 its fetch of a group overlaps the merge of the previous one, so DST
    lowers latency there; a setting is eligible only if its recall stays within
    0.002 of the throughput pick's (or at the target, when that is met)."""
    import torch
    from .groundtruth import recall_at_k
    dq = torch.from_numpy(np.ascontiguousarray(queries, dtype=np.float32)).cuda()
    prof = {}
    for ef in ef_list:
        # pilot at a large filter: visited count -> Bloom size
        _, r = _time_batch(index, dq, reps=1, k=k, ef=ef, cand_queue_size=min(256, max(32, ef // 4)), bloom_bits=22)
        vis = float(np.percentile(r.visited.cpu().numpy(), 90))
        bits_fp = bloom_bits_for(vis, fp_target)
        rows = []
        for cq in cq_grid:
            if cq > max(32, ef):
                continue
            for (mc, mg), bits in [(m, b) for m in mcmg_grid for b in sorted({bits_fp, max(16, bits_fp - 1)})]:
                p = dict(k=k, ef=ef, mc=mc, mg=mg, cand_queue_size=cq, bloom_bits=bits)
                ms, r = _time_batch(index, dq, **p)
                rec = recall_at_k(r.ids.cpu().numpy(), gt, k)
                rows.append(dict(p, ms=ms, qps=len(queries) / ms * 1e3, recall=rec))
                if log:
                    log("tune ef=%d cq=%d mc=%d mg=%d bits=%d: recall %.4f, %.0f QPS" % (ef, cq, mc, mg, bits, rec,
                                                                                       rows[-1]["qps"]))
        ok = [x for x in rows if x["recall"] >= recall_target]
        best = max(ok, key=lambda x: x["qps"]) if ok else max(rows, key=lambda x: (x["recall"], x["qps"]))
        params = {kk: best[kk] for kk in ("k", "ef", "mc", "mg", "cand_queue_size", "bloom_bits")}
        need = min(recall_target, best["recall"] - 0.002) if ok else best["recall"] - 0.002
        lat = {"inter": _time_single(index, dq, **params)}
        opts = {"inter": dict(params, mode="inter", channels=None)}
        lat_recall = {"inter": best["recall"]}
        for ch in latency_channels:
            for mc, mg in latency_mcmg:
                pc = dict(params, mc=mc, mg=mg, bloom_bits=channel_bloom_bits(params["bloom_bits"], ch))
                _, r = _time_batch(index, dq, reps=1, mode="intra", channels=ch, **pc)
                rec = recall_at_k(r.ids.cpu().numpy(), gt, k)
                name = "intra_%d_mc%d_mg%d" % (ch, mc, mg)
                if log:
                    log("tune latency %s ef=%d: recall %.4f (needs %.4f)" % (name, ef, rec, need))
                if rec < need:
                    continue
                lat[name] = _time_single(index, dq, mode="intra", channels=ch, **pc)
                opts[name] = dict(pc, mode="intra", channels=ch)
                lat_recall[name] = rec
        fastest = min(lat, key=lat.get)
        fp = opts[fastest]
        prof[profile_key(dim, degree, ef)] = {
            "throughput": {"params": dict(params, mode="inter"), "qps": best["qps"], "recall": best["recall"]},
            "latency": {"threads_per_query": 32 if fp["mode"] == "inter" else 32 * (12 // fp["channels"] * fp["channels"] + 1),
                        "mode": fp["mode"], "channels": fp["channels"], "bloom_bits": fp["bloom_bits"],
                        "mc": fp["mc"], "mg": fp["mg"], "recall": lat_recall[fastest],
                        "median_ms": lat},
            "visited_p90": vis, "recall_target_met": bool(ok), "grid": rows,
        }
    return prof


def best_for_recall(profile, recall_target):
    """The fastest throughput entry of a profile meeting the recall target (or
    the highest-recall one), as (key, entry)."""
    items = list(profile.items())
    ok = [(kk, v) for kk, v in items if v["throughput"]["recall"] >= recall_target]
    if ok:
        return max(ok, key=lambda kv: kv[1]["throughput"]["qps"])
    return max(items, key=lambda kv: kv[1]["throughput"]["recall"])


def save_profile(profile, path):
    old = load_profile(path) if os.path.exists(path) else {}
    old.update(profile)
    with open(path, "w") as f:
        json.dump(old, f, indent=1)


def load_profile(path):
    with open(path) as f:
        return json.load(f)


def pick(profile, dim, degree, ef, objective="throughput"):
    """Parameters for (dim, degree, ef) from a saved profile (nearest ef at or above)."""
    keys = [kk for kk in profile if kk.startswith("D%d_R%d_" % (dim, degree))]
    if not keys:
        raise KeyError("no profile for D=%d degree=%d" % (dim, degree))
    efs = sorted(int(kk.split("_ef")[1]) for kk in keys)
    e = next((x for x in efs if x >= ef), efs[-1])
    entry = profile[profile_key(dim, degree, e)]
    if objective == "throughput":
        return dict(entry["throughput"]["params"])
    p = dict(entry["throughput"]["params"])
    lat = entry["latency"]
    p["mode"] = lat["mode"]
    if lat["channels"]:
        p["channels"] = lat["channels"]
    for kk in ("bloom_bits", "mc", "mg"):
        if lat.get(kk):
            p[kk] = lat[kk]
    return p
