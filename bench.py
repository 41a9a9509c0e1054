"""Benchmark: QPS at recall@10 >= 0.95 (plus p50/p99 latency) of the graph
traversal path on B200, plain vs batched/served, against the reference's CPU
search on the host cores.

Headline (one GPU): the batched persistent kernel on a flat graph --
10M base vectors, D=128, integers round(|N(0,40)|) clipped to [0,255]
(seeded stand-in for SIFT10M), NSG-style single-layer graph of max degree 64
from the medoid built on the GPU (seed 1), 100k queries in ONE launch with ef
drawn from {32,64,128,256}, k from {1,10,100} and mc from {1,2,4} per query
(seeded).  A step is that launch with the queries resident in HBM; `e2e`
repeats it through the public API from pinned host buffers.  Recall is scored
against FP64 ground truth on the first 10k queries.  Beside it, the same
graph and queries at uniform k=10 and growing ef, to show where recall@10
reaches 0.95.

Extra keys (the other workloads, same run; --workloads selects them):
  sift100k_hnsw_m16: 100k x 128 sift-like, HNSW-style M=16 graph, 1000 queries,
        k=10, ef=64, mc=1
  deep1m_hnsw_m32: 1M x 96 unit-normal, HNSW-style M=32, 10k queries: throughput
        sweep to recall >= 0.95, batch-1 latency grid ef {64,128,256} x
        mc {1,2,4} (inter and intra), BF16/FP8 traversal + FP32 rerank, served
  sbert1m_hnsw_m32: 1M x 384 unit-normal, HNSW-style M=32, BF16 and FP8-E4M3
        traversal with FP32 rerank, ef {64,128}, mc=2, distance error vs FP64
  serving_sift10m_sbert1m: the sift10m and sbert1m indexes resident together,
        Poisson arrivals 10k-500k QPS, each request a random index, k, ef and
        mc; p50/p99 and sustained QPS

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--workloads sift100k,deep1m,sbert1m,serving]
       multi-GPU: python -m torch.distributed.run --nproc-per-node N bench.py --gpus N
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "falcon-accelerate-graph-vector-search_b200"))

RECALL_TARGET = 0.95
# deep1m_hnsw_m32: the operating point the autotuner selects at recall@10 >=
# 0.95 on this workload (recorded by the bench); --profile-throughput captures it
DEEP1M_THROUGHPUT_POINT = dict(k=10, ef=1024, mc=1, mg=1, cand_queue_size=256, bloom_bits=19)
METRIC = "QPS at recall@10>=0.95 (batched search; plain vs batched/served)"

# sift10m_nsg_r64: the headline workload
SIFT10M = dict(n=10_000_000, dim=128, nq=100_000, degree=64, seed_data=0, seed_query=1, seed_graph=1, ngt=10_000,
            efs=(32, 64, 128, 256), ks=(1, 10, 100), mcs=(1, 2, 4), cq=32, bits=16, param_seed=7,
            search_passes=((128, 1.0),))
WORKLOAD_SIFT10M = ("sift10m_nsg_r64: 10M x 128 clipped-integer base (seeded SIFT10M stand-in), NSG-style graph max degree 64 "
             "from the medoid (GPU-built, seed 1), 100k queries in one launch, per-query ef in {32,64,128,256}, "
             "k in {1,10,100}, mc in {1,2,4}")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [s.strip() for s in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(hops, visited, dim, degree, ks, efs=None, elem_bytes=4, scale_bytes=0, rerank=False):
    """Bytes each query must move, summed: its gathered vectors, its expanded
    adjacency rows (count word + max_degree ids), the query and its k results
    (id + distance); with a rerank the FP32 vectors of its ef candidates."""
    dpad = (dim + 15) // 16 * 16
    b = visited.astype(np.float64) * (dpad * elem_bytes + scale_bytes) + hops.astype(np.float64) * (4 + 4 * degree)
    b += dim * 4 + np.asarray(ks, dtype=np.float64) * 8
    if rerank:
        b += np.asarray(efs, dtype=np.float64) * dpad * 4
    return float(b.sum())


def distance_error_f64(x, q, ids, dists):
    """Relative error of returned distances against FP64 recomputation (same
    ids): max and mean over all valid results."""
    ids = np.asarray(ids)
    d = np.asarray(dists, dtype=np.float64)
    m = ids >= 0
    qq = np.repeat(np.arange(ids.shape[0]), ids.shape[1]).reshape(ids.shape)[m]
    diff = x[ids[m]].astype(np.float64) - q[qq].astype(np.float64)
    ref = (diff * diff).sum(1)
    rel = np.abs(d[m] - ref) / np.maximum(ref, 1e-30)
    return {"max_rel": float(rel.max()), "mean_rel": float(rel.mean())}


def timed(fn, reps=3):
    """Best CUDA-event time (ms) of fn() over reps, after one warm call; returns (ms, last result)."""
    import torch
    r = fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        a.record()
        r = fn()
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best, r


def batch1_latency(ix, dq, n, **p):
    """p50/p99 (ms) of one-query search calls, CUDA events around each call;
    the result tensors are allocated once (device_results) and reused."""
    import torch
    from falcon_b200.index import device_results
    out = device_results(1, int(p.get("k", 10)), device=dq.device)
    lat = []
    for i in range(n):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ix.search(dq[i:i + 1], out=out, **p)
        b.record()
        b.synchronize()
        lat.append(a.elapsed_time(b))
    lat = np.array(lat[min(10, n // 4):])
    return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))


def rounded(d):
    return {k: (round(v, 5) if isinstance(v, float) else v) for k, v in d.items()}


# ---------------------------------------------------------------------------
# sift10m_nsg_r64: data, graph, ground truth, mixed per-query parameters
# ---------------------------------------------------------------------------
def sift10m_params(nq):
    """Per-query (ef, k, mc) drawn by a seeded generator; ef is raised to k."""
    rng = np.random.default_rng(SIFT10M["param_seed"])
    efs = rng.choice(SIFT10M["efs"], nq)
    ks = rng.choice(SIFT10M["ks"], nq)
    mcs = rng.choice(SIFT10M["mcs"], nq)
    return np.maximum(efs, ks), ks, mcs


def sift10m_workload(dev, rank=0, timings=None):
    """Base, queries (seeded by rank for replicas), graph (host formats.Graph),
    FP64 ground truth (top 100) of the first ngt queries."""
    import torch
    from falcon_b200.groundtruth import shortlist_f64_tiled
    from falcon_b200.nsg import build_nsg
    from falcon_b200.synthetic import sift_like_blocks
    tm = timings if timings is not None else {}
    t = time.time()
    x = sift_like_blocks(SIFT10M["n"], SIFT10M["dim"], seed=SIFT10M["seed_data"])
    q = sift_like_blocks(SIFT10M["nq"], SIFT10M["dim"], seed=SIFT10M["seed_query"] + 1000 * rank)
    tm["data_s"] = time.time() - t
    cache = SIFT10M.get("graph_cache")
    if cache and os.path.exists(cache):
        # a graph and ground truth saved by an earlier run of the same workload (profiling runs)
        from falcon_b200.formats import Graph
        z = np.load(cache)
        st = json.loads(str(z["stats"]))
        g = Graph(x, z["links"], SIFT10M["degree"], int(z["entry"]))
        gt = z["gt"]
        tm["graph_cache"] = cache
        log("sift10m workload from %s" % cache)
        return x, q, g, gt, st
    xd = torch.from_numpy(x).to(dev)
    st = {}
    t = time.time()
    g = build_nsg(x, SIFT10M["degree"], seed=SIFT10M["seed_graph"], search_passes=SIFT10M["search_passes"], device=dev,
                  vectors_device=xd, stats=st, verbose=True)
    tm["graph_s"] = time.time() - t
    t = time.time()
    gt, _ = shortlist_f64_tiled(x, q[:SIFT10M["ngt"]], 100, shortlist=128, base_device=xd, device=dev)
    tm["ground_truth_s"] = time.time() - t
    if cache:
        np.savez(cache, links=g.links, entry=g.entry_point, gt=gt, stats=json.dumps(st))
    del xd
    torch.cuda.empty_cache()
    log("sift10m workload: %s" % rounded(tm))
    return x, q, g, gt, st


def mixed_recall(ids, gt, ks):
    """recall@10 over the queries with k >= 10 (first 10 results against the
    10 true nearest), recall@1 over k = 1, recall@100 over k = 100."""
    from falcon_b200.groundtruth import recall_at_k
    n = len(gt)
    ids, ks = np.asarray(ids)[:n], np.asarray(ks)[:n]
    out = {}
    m10 = ks >= 10
    if m10.any():
        out["recall@10_k>=10"] = recall_at_k(ids[m10], gt[m10], 10)
    m1 = ks == 1
    if m1.any():
        out["recall@1_k=1"] = recall_at_k(ids[m1], gt[m1], 1)
    m100 = ks == 100
    if m100.any():
        out["recall@100_k=100"] = recall_at_k(ids[m100], gt[m100], 100)
    out["queries_scored"] = int(n)
    return out


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def headline_sift10m(args, dev, local, rank, ws, out):
    import torch
    from falcon_b200 import FalconIndex, make_params
    from falcon_b200.index import params_array
    tm = {}
    x, q, g, gt, gstats = sift10m_workload(dev, rank, tm)
    t = time.time()
    ix = FalconIndex(g, device=local)
    tm["index_s"] = time.time() - t
    nq = len(q)
    efs, ks, mcs = sift10m_params(nq)
    parr = params_array([make_params(k=int(k), ef=int(e), mc=int(m), mg=1, cand_queue_size=SIFT10M["cq"],
                                     bloom_bits=SIFT10M["bits"]) for e, k, m in zip(efs, ks, mcs)])
    dq = torch.from_numpy(q).to(dev)
    for _ in range(args.warmup):
        r = ix.search(dq, per_query=parr)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.profile_region:
        torch.cuda.profiler.start()
    with ClockSampler(local) as clk:
        ev0.record()
        for _ in range(args.steps):
            r = ix.search(dq, per_query=parr)
        ev1.record()
        torch.cuda.synchronize()
    if args.profile_region:
        torch.cuda.profiler.stop()
    ms = ev0.elapsed_time(ev1)
    if ws > 1:
        tt = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms = float(tt.item())
        torch.distributed.barrier()
    ms_step = ms / args.steps
    ids = r.ids.cpu().numpy()
    hops, vis = r.hops.cpu().numpy(), r.visited.cpu().numpy()
    rec = mixed_recall(ids, gt, ks)
    log("sift10m headline: %.2f ms/step, %.0f QPS, %s, hops %.1f visited %.1f" % (
        ms_step, nq / ms_step * 1e3, rounded(rec), hops.mean(), vis.mean()))
    if args.profile_region:
        print(json.dumps({"profiled_steps": args.steps, "search": "sift10m mixed", "ms_per_step": ms_step,
                          "n_base": SIFT10M["n"], "queries_per_step": nq, "hops_mean": float(hops.mean()),
                          "visited_mean": float(vis.mean()),
                          "bytes_per_query": algorithmic_bytes(hops, vis, SIFT10M["dim"], SIFT10M["degree"], ks) / nq}))
        ix.close()
        return None

    # end to end through the public API: pinned host queries, results into
    # pinned host arrays allocated once (as the reference host allocates its
    # result buffers once)
    from falcon_b200.index import pinned_results
    qh = torch.from_numpy(q).pin_memory().numpy()
    outh = pinned_results(nq, int(ks.max()))
    e2e = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        rh = ix.search(qh, per_query=parr, out=outh)
        if i >= args.warmup:
            e2e.append(time.perf_counter() - t)
    e2e_ms = sum(e2e) / len(e2e) * 1e3
    if ws > 1:
        tt = torch.tensor([e2e_ms], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    same = bool(np.array_equal(rh.ids, ids) and np.array_equal(rh.hops, hops))

    peak, peak_kind = measured_peak()
    alg = algorithmic_bytes(hops, vis, SIFT10M["dim"], SIFT10M["degree"], ks)
    achieved = alg / (ms_step / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "peak_kind": peak_kind, "bytes_per_query": alg / nq,
            "kernel": "inter_kernel<f32, EPL=8, VROWS=1>",
            "achieved_from": "algorithmic bytes of the step / CUDA-event step time (the search kernel is the "
                             "step's only kernel)"}
    traffic_from_profile(roof, "sift10m_mixed", alg)
    out.update({
        "metric": METRIC, "value": ws * nq / (ms_step / 1e3), "unit": "queries/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded clipped-integer stand-in for SIFT10M; the reference's datasets are not available)",
        "config": {"workload": WORKLOAD_SIFT10M, "queries_per_step": nq, "per_query": "ef/k/mc drawn per query (seed 7), "
                   "ef raised to k, cand_queue_size 32, bloom_bits 16, mg 1 (the reference defaults)",
                   "mode": "inter", "recall": rec, "recall_target_reached": bool(rec.get("recall@10_k>=10", 0) >=
                                                                             RECALL_TARGET),
                   "hops_mean": float(hops.mean()), "visited_mean": float(vis.mean()),
                   "graph": {k: v for k, v in gstats.items() if not k.endswith("_s")},
                   "graph_build_s": round(gstats.get("build_s", 0.0), 1), "timings_s": rounded(tm),
                   "parallelism": "replicas" if ws > 1 else "single",
                   "l2": "inputs larger than L2 (5.1 GB vectors + 3.2 GB links vs 126 MB L2)"},
        "e2e": {"value": ws * nq / (e2e_ms / 1e3), "unit": "queries/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(q.nbytes + nq * 48),
                "d2h_bytes_per_step": int(nq * int(ks.max()) * 8 + nq * 8),
                "results_equal_device_run": same},
        "gpu_launches": args.steps,   # one search kernel per step (no upper layers on this graph)
        "clocks": clk.summary(),
        "roofline": roof,
    })
    return dict(ix=ix, x=x, q=q, g=g, gt=gt, dq=dq, parr=parr, efs=efs, ks=ks, mcs=mcs, ids=ids,
                dists=r.dists.cpu().numpy(), hops=hops, vis=vis)


def traffic_from_profile(roof, key, alg_bytes):
    """DRAM traffic per launch from the ncu capture recorded in
    profiles/traffic.json, used only while it was taken on the current kernel
    source (the file records the source's hash)."""
    import hashlib
    tp = os.path.join(REPO, "profiles", "traffic.json")
    if not os.path.exists(tp):
        return
    tr = json.load(open(tp))
    e = tr.get(key)
    src = os.path.join(REPO, "falcon-accelerate-graph-vector-search_b200", "csrc", "falcon_kernels.cu")
    h = hashlib.sha256(open(src, "rb").read()).hexdigest()[:16]
    if not e or e.get("kernel_source_sha16") != h:
        roof["traffic_note"] = "no ncu capture of the current kernel source for this workload"
        return
    roof["traffic"] = e["ratio"] * alg_bytes
    roof["traffic_ratio"] = e["ratio"]
    roof["traffic_note"] = e["note"]


def recall_curve_sift10m(H, out):
    """Same graph and the ground-truth queries at uniform k=10 and growing ef:
    the smallest ef whose recall@10 reaches the target, or the best reached."""
    import torch
    from falcon_b200.groundtruth import recall_at_k
    ix, dq, gt = H["ix"], H["dq"], H["gt"]
    n = len(gt)
    pts = []
    for ef, cq, bits, mc, mg in ((64, 32, 16, 1, 1), (256, 32, 16, 1, 1), (256, 64, 18, 2, 4), (512, 128, 18, 1, 1),
                                 (1024, 256, 20, 1, 1), (1024, 256, 20, 2, 4)):
        ms, r = timed(lambda: ix.search(dq[:n], k=10, ef=ef, mc=mc, mg=mg, cand_queue_size=cq, bloom_bits=bits), 2)
        rec = recall_at_k(r.ids.cpu().numpy(), gt, 10)
        pts.append(dict(ef=ef, cq=cq, bits=bits, mc=mc, mg=mg, recall=rec, qps=n / ms * 1e3,
                        visited=float(r.visited.float().mean()), hops=float(r.hops.float().mean())))
        log("sift10m uniform k=10: %s" % rounded(pts[-1]))
    ok = [p for p in pts if p["recall"] >= RECALL_TARGET]
    best = min(ok, key=lambda p: (p["ef"], -p["qps"])) if ok else max(pts, key=lambda p: p["recall"])
    out["sift10m_uniform_k10"] = {"queries": n, "points": [rounded(p) for p in pts], "selected": rounded(best),
                               "recall_target_reached": bool(ok),
                               "note": "i.i.d. coordinates give full intrinsic dimension (128): graph search needs "
                                       "a large ef on this stand-in; the kernel's ef limit is 1024"}


def cpu_baselines_sift10m(H, out, threads, budget_s=15.0):
    """Reference CPU search (the reference's vendored hnswlib, built from its
    headers) on the same graph from the same medoid with the same per-query ef
    and k, all host threads, bounded sample; then the oracle (the C
    restatement of the FPGA traversal) on a smaller sample, whose results are
    also compared bit for bit with the GPU's rows for the same queries."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    g, q, gt = H["g"], H["q"], H["gt"]
    efs, ks, mcs = H["efs"], H["ks"], H["mcs"]
    res = {}
    if oracle.Hnsw.available():
        t = time.time()
        h = oracle.Hnsw.from_graph(g.vectors, g.adjacency(), g.entry_point)
        load_s = time.time() - t
        n = min(len(gt), 2000)
        t = time.time()
        h.search_mixed(q[:n], ks[:n], efs[:n], threads)
        dt = time.time() - t
        reps = int(max(1, min(10, budget_s / max(dt, 1e-3))))
        n = int(min(len(gt), max(n, n * reps)))
        t = time.time()
        lab, _ = h.search_mixed(q[:n], ks[:n], efs[:n], threads)
        dt = time.time() - t
        h.free()
        res["cpu_baseline"] = {"value": n / dt, "unit": "queries/s", "cores": threads, "kind": "reference",
                               "isa": oracle.Hnsw.isa(), "cpu": oracle.Hnsw.cpu_model(),
                               "sample": "first %d of the 100k queries, hnswlib searchKnn with each query's ef and k "
                                         "(setEf per (ef, k) group), base layer from the same medoid; mc has no "
                                         "hnswlib counterpart" % n,
                               "recall": mixed_recall(lab, gt[:n], ks[:n]), "graph_load_s": load_s}
        log("sift10m cpu baseline: %s" % rounded({k: v for k, v in res["cpu_baseline"].items() if k != "recall"}))
    # oracle port + parity sample
    og = oracle.OracleGraph(g.vectors, g.links, g.max_degree, g.ids_offset)
    m = min(len(q), 4 * threads)
    plist = [oracle.make_params(k=int(k), ef=int(e), mc=int(c), mg=1, cand_queue_size=SIFT10M["cq"],
                                bloom_bits=SIFT10M["bits"]) for e, k, c in zip(efs[:m], ks[:m], mcs[:m])]
    t = time.time()
    ids, d, hops, vis, _ = oracle.search(og, q[:m], g.entry_point, plist, out_stride=H["ids"].shape[1],
                                         threads=threads)
    dt = time.time() - t
    exact = [bool(np.array_equal(ids[i], H["ids"][i]) and np.array_equal(d[i].view(np.uint32),
                                                                         H["dists"][i].view(np.uint32))
                  and hops[i] == H["hops"][i] and vis[i] == H["vis"][i]) for i in range(m)]
    # the same restatement on one core (a few queries)
    m1 = min(m, 8)
    t = time.time()
    oracle.search(og, q[:m1], g.entry_point, plist[:m1], out_stride=H["ids"].shape[1], threads=1)
    dt1 = time.time() - t
    res["cpu_fpga_semantics_port"] = {"value": m / dt, "unit": "queries/s", "cores": threads, "kind": "port",
                                      "sample": "first %d queries, oracle (C restatement of the FPGA traversal) with "
                                                "the GPU's per-query parameters" % m,
                                      "single_core": {"value": m1 / dt1, "unit": "queries/s", "cores": 1,
                                                      "sample": "first %d queries" % m1}}
    res["parity_sample"] = {"queries": m, "bit_exact": int(sum(exact)),
                            "compared": "ids, distance bits, hops, visited of the GPU headline rows against the "
                                        "oracle on the same 10M graph"}
    log("sift10m parity sample: %d/%d bit-exact; oracle %.1f QPS" % (sum(exact), m, m / dt))
    del og
    return res


def run_deep1m(args, dev, local, out):
    """deep1m_hnsw_m32: 1M x 96 unit-normal, HNSW-style M=32; throughput at the
    recall target, batch-1 latency grid, reduced precision + rerank, served."""
    import torch
    from falcon_b200 import FalconIndex
    from falcon_b200.autotune import channel_bloom_bits
    from falcon_b200.graph import build_graph, build_upper_layers
    from falcon_b200.groundtruth import recall_at_k, shortlist_f64
    from falcon_b200.synthetic import unit_normal
    n, dim, nq, k = args.deep1m_n, 96, 10_000, 10
    t0 = time.time()
    x = unit_normal(n, dim, seed=0)
    q = unit_normal(nq, dim, seed=1)
    g = build_graph(x, 64, device=dev)
    upper = build_upper_layers(x, 32, seed=0, device=dev)
    gt, _ = shortlist_f64(x, q, k, device=dev)
    ix = FalconIndex(g, storage=("f32", "bf16", "fp8"), device=local)
    ix.set_upper_layers(upper)
    dq = torch.from_numpy(q).to(dev)
    build_s = time.time() - t0
    # operating point from the autotuner (falcon_b200.autotune): per ef, Bloom
    # size from the visited count, then candidate queue and (mc, mg) for
    # throughput at the recall target, on a 2000-query sample
    from falcon_b200.autotune import best_for_recall, pick, tune
    prof = tune(ix, q[:2000], gt[:2000], dim, 64, ef_list=(256, 512, 1024), k=k, recall_target=RECALL_TARGET,
                cq_grid=(64, 256), mcmg_grid=((1, 1), (2, 4), (1, 4)), latency_channels=(4,),
                log=lambda m: log("deep1m " + m))
    key, entry = best_for_recall(prof, RECALL_TARGET)
    P = pick(prof, dim, 64, entry["throughput"]["params"]["ef"])
    P.pop("mode", None)
    ef, mc, mg, cq, bits = P["ef"], P["mc"], P["mg"], P["cand_queue_size"], P["bloom_bits"]
    ms, r = timed(lambda: ix.search(dq, **P), 3)
    sel = dict(ef=ef, mc=mc, mg=mg, cq=cq, bits=bits, recall=recall_at_k(r.ids.cpu().numpy(), gt, k),
               qps=nq / ms * 1e3, ms=ms, hops=float(r.hops.float().mean()), visited=float(r.visited.float().mean()),
               profile_key=key)
    ok = sel["recall"] >= RECALL_TARGET
    pts = [rounded({kk: v for kk, v in row.items()}) for e in prof.values() for row in e["grid"]]
    log("deep1m selected by the autotuner: %s" % rounded(sel))
    ms_b, rb = timed(lambda: ix.search(dq, precision="bf16", rerank=True, **P))
    ms_f, rf = timed(lambda: ix.search(dq, precision="fp8", rerank=True, **P))
    # roofline of the throughput point: algorithmic bytes of each launch over
    # its CUDA-event time (the descent kernel is < 1 % of the step)
    peak, peak_kind = measured_peak()
    roof1 = {}
    for name, res, t_ms, eb, sb, rr in (("f32", r, ms, 4, 0, False), ("bf16_rerank", rb, ms_b, 2, 0, True),
                                        ("fp8_rerank", rf, ms_f, 1, 4, True)):
        alg = algorithmic_bytes(res.hops.cpu().numpy(), res.visited.cpu().numpy(), dim, 64, np.full(nq, k),
                                np.full(nq, ef), elem_bytes=eb, scale_bytes=sb, rerank=rr)
        gbs = alg / (t_ms / 1e3) / 1e9
        roof1[name] = {"achieved_gbs": gbs, "frac": gbs / peak, "bytes_per_query": alg / nq}
    if all(P.get(kk) == v for kk, v in DEEP1M_THROUGHPUT_POINT.items()):
        traffic_from_profile(roof1["f32"], "deep1m_f32_throughput_point", roof1["f32"]["bytes_per_query"] * nq)
    roof1["peak_gbs"] = peak
    roof1["peak_kind"] = peak_kind
    roof1["note"] = ("latency-bound: 3 blocks of 4 warps per SM (registers, and the ef-1024 result list in shared "
                     "memory) and per-warp 2^19-bit filters in global memory (113 MB, near the L2 size)")
    r = ix.search(dq, **P)
    derr = {"f32": distance_error_f64(x, q, r.ids.cpu().numpy(), r.dists.cpu().numpy())}
    for prec, res in (("bf16", rb), ("fp8", rf)):
        raw = ix.search(dq, precision=prec, **P)
        derr[prec + "_rerank"] = distance_error_f64(x, q, res.ids.cpu().numpy(), res.dists.cpu().numpy())
        derr[prec + "_traversal"] = distance_error_f64(x, q, raw.ids.cpu().numpy(), raw.dists.cpu().numpy())
        derr[prec + "_traversal"]["recall@10"] = recall_at_k(raw.ids.cpu().numpy(), gt, k)
    # batch-1 latency grid (ef {64,128,256} x mc {1,2,4}), inter and intra (4 channels)
    grid = []
    for ef_l in (64, 128, 256):
        for mc_l in (1, 2, 4):
            row = {"ef": ef_l, "mc": mc_l}
            for mode, extra in (("inter", {}), ("intra4", dict(mode="intra", channels=4)),
                                ("intra4_mg4", dict(mode="intra", channels=4, mg=4))):
                pl = dict(k=k, ef=ef_l, mc=mc_l, mg=1, cand_queue_size=32, bloom_bits=16)
                pl.update(extra)
                p50, p99 = batch1_latency(ix, dq, args.latency_samples, **pl)
                rr = ix.search(dq[:2000], **pl)
                row[mode] = {"p50_ms": p50, "p99_ms": p99, "recall@10": recall_at_k(rr.ids.cpu().numpy(), gt[:2000], k)}
            grid.append(row)
            log("deep1m batch-1 %s" % row)
    # batch-1 at the throughput operating point
    lat_sel = {}
    for mode, extra in (("inter", {}), ("intra4", dict(mode="intra", channels=4,
                                                       bloom_bits=channel_bloom_bits(bits, 4)))):
        pl = dict(P)
        pl.update(extra)
        p50, p99 = batch1_latency(ix, dq, args.latency_samples, **pl)
        lat_sel[mode] = {"p50_ms": p50, "p99_ms": p99}
    # the autotuner's latency pick at the same ef: mode, channels and the DST
    # setting (mc, mg) whose recall stays at the target
    PL = pick(prof, dim, 64, ef, objective="latency")
    if PL.get("channels") is None:
        PL.pop("channels", None)
    p50, p99 = batch1_latency(ix, dq, args.latency_samples, **PL)
    rl = ix.search(dq, **PL)
    lat_sel["tuned"] = {"p50_ms": p50, "p99_ms": p99, "recall@10": recall_at_k(rl.ids.cpu().numpy(), gt, k),
                        "params": {kk: v for kk, v in PL.items() if kk != "k"}}
    log("deep1m batch-1 at the operating point: %s" % lat_sel)
    served = None if args.no_serve else serve_deep1m(ix, q, gt, prof, ef, nq / (ms_b / 1e3))
    ix.close()
    out["deep1m_hnsw_m32"] = {
        "workload": "deep1m_hnsw_m32: 1M x 96 unit-normal (seeded Deep1M stand-in), HNSW-style M=32 graph (exact "
                    "kNN + hnswlib's neighbour heuristic + reverse edges, upper layers with hnswlib's level "
                    "distribution), 10k queries, k=10; searches descend the upper layers",
        "n_base": n, "build_s": build_s, "autotuner_grid": pts, "selected": rounded(sel),
        "recall_target_reached": bool(ok),
        "latency_pick": {kk: v for kk, v in entry["latency"].items()},
        "bf16_rerank": {"value": nq / (ms_b / 1e3), "unit": "queries/s",
                        "recall@10": recall_at_k(rb.ids.cpu().numpy(), gt, k)},
        "fp8_rerank": {"value": nq / (ms_f / 1e3), "unit": "queries/s",
                       "recall@10": recall_at_k(rf.ids.cpu().numpy(), gt, k)},
        "roofline": roof1,
        "distance_error_vs_f64": derr, "latency_batch1_grid": grid, "latency_batch1_selected": lat_sel,
        "served": served}


def serve_deep1m(ix, q, gt, prof, ef, batched_bf16_qps):
    """Continuous batching of single-query requests (BF16 traversal + exact
    FP32 rerank) with Poisson arrivals at 50 %, 80 % of the batched BF16 rate
    and at saturation; each request's parameters come from the autotuner's
    profile for its ef (FalconServer.auto_params)."""
    from falcon_b200.groundtruth import recall_at_k
    from falcon_b200.serving import FalconServer, poisson_arrivals
    k = 10
    sv = FalconServer(ring_capacity=65536, max_k=k, ef_max=ef, cand_queue_max=256, bloom_bits_max=20, mc_max=4,
                      mg_max=4, dim_max=96, idle_exit_us=5000)
    iid = sv.add_index(ix)
    sv.set_profile(prof)
    p = sv.auto_params(iid, k=k, ef=ef, precision="bf16", rerank=True)
    n = 2 * len(q)
    qq = np.concatenate([q, q])
    out = {"precision": "bf16+fp32 rerank", "requests_per_point": n, "points": [],
           "entry": "each request descends the HNSW upper layers"}
    sv.replay(np.full(1000, iid), qq[:1000], p, poisson_arrivals(1000, batched_bf16_qps, 9), k)
    for frac in (0.5, 0.8, 10.0):
        rate = batched_bf16_qps * frac
        arr = poisson_arrivals(n, rate, seed=int(frac * 100))
        lat, ids, d, hops, vis, el = sv.replay(np.full(n, iid), qq, p, arr, k)
        pt = {"offered_qps": rate if frac < 10 else None,
              "offered": "saturation" if frac >= 10 else "%.0f%%" % (frac * 100),
              "sustained_qps": n / (el / 1e6), "p50_ms": float(np.percentile(lat, 50)) / 1e3,
              "p99_ms": float(np.percentile(lat, 99)) / 1e3, "recall@10": recall_at_k(ids[:len(q)], gt, k)}
        log("deep1m served %s" % rounded(pt))
        out["points"].append(pt)
    sv.close()
    return out


def run_sift100k(args, dev, local, out, threads):
    """sift100k_hnsw_m16: 100k x 128 sift-like, HNSW-style M=16 (degree 32), 1000
    queries, k=10, ef=64, mc=1; hnswlib on the same graph beside it."""
    import torch
    from falcon_b200 import FalconIndex
    from falcon_b200.graph import build_graph, build_upper_layers
    from falcon_b200.groundtruth import brute_force_f64, recall_at_k
    from falcon_b200.synthetic import sift_like
    x = sift_like(100_000, 128, seed=0)
    q = sift_like(1000, 128, seed=1)
    t = time.time()
    g = build_graph(x, 32, device=dev)
    upper = build_upper_layers(x, 16, seed=0, device=dev)
    build_s = time.time() - t
    gt, _ = brute_force_f64(x, q, 10)
    ix = FalconIndex(g, device=local)
    ix.set_upper_layers(upper)
    dq = torch.from_numpy(q).to(dev)
    P = dict(k=10, ef=64, mc=1, mg=1, cand_queue_size=32, bloom_bits=16)
    ms, r = timed(lambda: ix.search(dq, **P), 5)
    p50, p99 = batch1_latency(ix, dq, min(args.latency_samples, 1000), **P)
    res = {"workload": "sift100k_hnsw_m16: 100k x 128 clipped-integer base, HNSW-style M=16 (degree-32 base layer, "
                       "upper layers), 1000 queries, k=10, ef=64, mc=1, cand queue 32, 2^16-bit filter",
           "value": len(q) / ms * 1e3, "unit": "queries/s", "recall@10": recall_at_k(r.ids.cpu().numpy(), gt, 10),
           "hops_mean": float(r.hops.float().mean()), "visited_mean": float(r.visited.float().mean()),
           "latency_batch1": {"p50_ms": p50, "p99_ms": p99}, "build_s": build_s,
           "l2": "the 51 MB base fits in L2: no HBM-roofline claim on this workload"}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle
        if oracle.Hnsw.available():
            h = oracle.Hnsw.from_graph(x, g.adjacency(), g.entry_point)
            h.set_upper(upper)
            h.search(q, 10, 64, threads)
            t = time.time()
            lab, _ = h.search(q, 10, 64, threads)
            dt = time.time() - t
            res["cpu_baseline"] = {"value": len(q) / dt, "unit": "queries/s", "cores": threads, "kind": "reference",
                                   "isa": oracle.Hnsw.isa(), "recall@10": recall_at_k(lab, gt, 10),
                                   "sample": "the 1000 queries, hnswlib searchKnn setEf(64) on the same graph with "
                                             "the same upper layers"}
            h.free()
    ix.close()
    log("sift100k: %s" % rounded({k2: v for k2, v in res.items() if not isinstance(v, dict)}))
    out["sift100k_hnsw_m16"] = res


def run_sbert1m(args, dev, local, out, keep=False):
    """sbert1m_hnsw_m32: 1M x 384 unit-normal, HNSW-style M=32, BF16 and FP8-E4M3
    (+ per-vector scale) traversal with FP32 accumulation and an exact FP32
    rerank of the final ef; ef {64,128}, mc=2, 10k queries."""
    import torch
    from falcon_b200 import FalconIndex
    from falcon_b200.graph import build_graph, build_upper_layers
    from falcon_b200.groundtruth import recall_at_k, shortlist_f64
    from falcon_b200.synthetic import unit_normal_blocks
    n, dim, nq = args.sbert1m_n, 384, 10_000
    t = time.time()
    x = unit_normal_blocks(n, dim, seed=3)
    q = unit_normal_blocks(nq, dim, seed=4)
    g = build_graph(x, 64, device=dev)
    upper = build_upper_layers(x, 32, seed=0, device=dev)
    gt, _ = shortlist_f64(x, q, 10, device=dev)
    ix = FalconIndex(g, storage=("f32", "bf16", "fp8"), device=local)
    ix.set_upper_layers(upper)
    build_s = time.time() - t
    dq = torch.from_numpy(q).to(dev)
    pts = []
    for ef in (64, 128):
        P = dict(k=10, ef=ef, mc=2, mg=1, cand_queue_size=32, bloom_bits=16)
        ms32, r32 = timed(lambda: ix.search(dq, **P))
        ids32 = r32.ids.cpu().numpy()
        row = {"ef": ef, "mc": 2, "f32": {"value": nq / ms32 * 1e3, "recall@10": recall_at_k(ids32, gt, 10),
                                          "distance_error_vs_f64": distance_error_f64(x, q, ids32, r32.dists.cpu().numpy())}}
        for prec in ("bf16", "fp8"):
            ms, rr = timed(lambda: ix.search(dq, precision=prec, rerank=True, **P))
            raw = ix.search(dq, precision=prec, **P)
            ids = rr.ids.cpu().numpy()
            hops, vis = rr.hops.cpu().numpy(), rr.visited.cpu().numpy()
            alg = algorithmic_bytes(hops, vis, dim, 64, np.full(nq, 10), np.full(nq, ef),
                                    elem_bytes=2 if prec == "bf16" else 1, scale_bytes=4 if prec == "fp8" else 0,
                                    rerank=True)
            row[prec + "_rerank"] = {
                "value": nq / ms * 1e3, "recall@10": recall_at_k(ids, gt, 10),
                "recall_vs_f32_path": float(np.mean([len(np.intersect1d(a, b)) / 10.0 for a, b in zip(ids, ids32)])),
                "distance_error_vs_f64": distance_error_f64(x, q, ids, rr.dists.cpu().numpy()),
                "traversal_distance_error_vs_f64": distance_error_f64(x, q, raw.ids.cpu().numpy(),
                                                                      raw.dists.cpu().numpy()),
                "roofline_achieved_gbs": alg / (ms / 1e3) / 1e9}
        pts.append(row)
        log("sbert1m %s" % json.dumps(row)[:600])
    out["sbert1m_hnsw_m32"] = {"workload": "sbert1m_hnsw_m32: 1M x 384 unit-normal (seeded SBERT1M stand-in), HNSW-style M=32, "
                               "10k queries, k=10, mc=2, cand queue 32, 2^16-bit filter; BF16 / FP8-E4M3 + per-vector "
                               "FP32 scale traversal, FP32 accumulation, exact FP32 rerank of the final ef",
                   "n_base": n, "build_s": build_s, "points": pts}
    if keep:
        return dict(ix=ix, q=q, x=x)
    ix.close()
    return None


def run_serving(args, H2, H3, out):
    """Online serving: the sift10m_nsg_r64 (FP32, D=128, NSG) and
    sbert1m_hnsw_m32 (BF16 + FP32 rerank, D=384, HNSW) indexes resident
    together; Poisson arrivals,
    each request a random index with k from {1,10,100}, ef from {32..256},
    mc from {1,2,4}."""
    from falcon_b200 import make_params
    from falcon_b200.serving import FalconServer, poisson_arrivals
    sv = FalconServer(ring_capacity=65536, max_k=100, ef_max=256, cand_queue_max=32, bloom_bits_max=16, mc_max=4,
                      mg_max=1, dim_max=384, idle_exit_us=5000)
    i2 = sv.add_index(H2["ix"])
    i3 = sv.add_index(H3["ix"])
    rng = np.random.default_rng(11)
    n = 40_000
    which = rng.integers(0, 2, n)
    ks = rng.choice([1, 10, 100], n)
    efs = np.maximum(rng.choice([32, 64, 128, 256], n), ks)
    mcs = rng.choice([1, 2, 4], n)
    q2, q3 = H2["q"], H3["q"]
    qmax = np.zeros((n, 384), dtype=np.float32)
    idx = rng.integers(0, 10_000, n)
    params, iids = [], np.where(which == 0, i2, i3).astype(np.int32)
    for i in range(n):
        if which[i] == 0:
            qmax[i, :128] = q2[idx[i]]
            params.append(make_params(k=int(ks[i]), ef=int(efs[i]), mc=int(mcs[i])))
        else:
            qmax[i] = q3[idx[i]]
            params.append(make_params(k=int(ks[i]), ef=int(efs[i]), mc=int(mcs[i]), precision="bf16", rerank=True))
    pts = []
    sv.replay(iids[:2000], qmax[:2000], params[:2000], poisson_arrivals(2000, 20000, 5), 100)
    for rate in (10_000, 50_000, 100_000, 200_000, 500_000):
        m = min(n, max(4000, int(rate * 0.25)))
        arr = poisson_arrivals(m, rate, seed=rate)
        lat, ids, d, hops, vis, el = sv.replay(iids[:m], qmax[:m], params[:m], arr, 100)
        pt = {"offered_qps": rate, "requests": m, "sustained_qps": m / (el / 1e6),
              "p50_ms": float(np.percentile(lat, 50)) / 1e3, "p99_ms": float(np.percentile(lat, 99)) / 1e3,
              "p50_ms_sift10m": float(np.percentile(lat[which[:m] == 0], 50)) / 1e3,
              "p50_ms_sbert1m": float(np.percentile(lat[which[:m] == 1], 50)) / 1e3}
        log("serving %s" % rounded(pt))
        pts.append(pt)
    inf = sv.info()
    sv.close()
    out["serving_sift10m_sbert1m"] = {"workload": "online serving: sift10m_nsg_r64 (FP32) and sbert1m_hnsw_m32 (BF16 + FP32 rerank) "
                               "resident together, Poisson arrivals, each request a random index, k {1,10,100}, "
                               "ef {32,64,128,256} (raised to k), mc {1,2,4}",
                   "points": pts, "kernel_launches": int(inf.kernel_launches)}


def profile_latency(args):
    """Batch-1 intra-query searches of deep1m_hnsw_m32 (1M x 96) at the DST latency
    point (ef 1024, mc 2, mg 4, 4 channels), bracketed by
    cudaProfilerStart/Stop, for a capture of intra_kernel; prints one line."""
    import torch
    from falcon_b200 import FalconIndex
    from falcon_b200.graph import build_graph, build_upper_layers
    from falcon_b200.synthetic import unit_normal
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = "cuda:%d" % local
    x = unit_normal(args.deep1m_n, 96, seed=0)
    q = unit_normal(64, 96, seed=1)
    g = build_graph(x, 64, device=dev)
    upper = build_upper_layers(x, 32, seed=0, device=dev)
    ix = FalconIndex(g, device=local)
    ix.set_upper_layers(upper)
    dq = torch.from_numpy(q).to(dev)
    P = dict(k=10, ef=1024, mc=2, mg=4, cand_queue_size=256, bloom_bits=18, mode="intra", channels=4)
    for i in range(args.warmup):
        ix.search(dq[i:i + 1], **P)
    torch.cuda.synchronize()
    lat = []
    torch.cuda.profiler.start()
    for i in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        r = ix.search(dq[i:i + 1], **P)
        b.record()
        b.synchronize()
        lat.append(a.elapsed_time(b))
    torch.cuda.profiler.stop()
    print(json.dumps({"profiled_searches": args.steps, "search": "deep1m batch-1 intra DST", "params": P,
                      "p50_ms": float(np.median(lat)), "hops_last": int(r.hops[0]), "visited_last": int(r.visited[0])}))
    ix.close()
    return 0


def profile_throughput(args):
    """deep1m_hnsw_m32 (1M x 96) 10k-query searches at the throughput point the
    tuner selects at recall 0.95 (ef 1024, cand queue 256, 2^19-bit filters,
    mc 1, mg 1), bracketed by cudaProfilerStart/Stop, for a DRAM capture of
    the inter kernel; prints one line."""
    import torch
    from falcon_b200 import FalconIndex
    from falcon_b200.graph import build_graph, build_upper_layers
    from falcon_b200.synthetic import unit_normal
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = "cuda:%d" % local
    nq = 10_000
    x = unit_normal(args.deep1m_n, 96, seed=0)
    q = unit_normal(nq, 96, seed=1)
    g = build_graph(x, 64, device=dev)
    upper = build_upper_layers(x, 32, seed=0, device=dev)
    ix = FalconIndex(g, device=local)
    ix.set_upper_layers(upper)
    dq = torch.from_numpy(q).to(dev)
    P = dict(DEEP1M_THROUGHPUT_POINT)
    for _ in range(args.warmup):
        r = ix.search(dq, **P)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.profiler.start()
    a.record()
    for _ in range(args.steps):
        r = ix.search(dq, **P)
    b.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    hops, vis = r.hops.cpu().numpy(), r.visited.cpu().numpy()
    alg = algorithmic_bytes(hops, vis, 96, 64, np.full(nq, P["k"]))
    print(json.dumps({"profiled_steps": args.steps, "search": "deep1m throughput point", "params": P,
                      "ms_per_step": a.elapsed_time(b) / args.steps, "hops_mean": float(hops.mean()),
                      "visited_mean": float(vis.mean()), "bytes_per_query": alg / nq}))
    ix.close()
    return 0


def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = "cuda:%d" % local
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    threads = os.cpu_count() or 1
    wl = {w.strip() for w in args.workloads.split(",") if w.strip()}
    out = {}
    t0 = time.time()
    H2 = headline_sift10m(args, dev, local, rank, ws, out)
    if H2 is None:
        return 0
    if ws == 1:
        recall_curve_sift10m(H2, out)
        if not args.no_cpu_baseline:
            res = cpu_baselines_sift10m(H2, out, threads)
            out["cpu_baseline"] = res.get("cpu_baseline")
            out["cpu_fpga_semantics_port"] = res.get("cpu_fpga_semantics_port")
            out["config"]["parity_sample"] = res.get("parity_sample")
        log("sift10m done at %.0fs" % (time.time() - t0))
        H3 = None
        if "sbert1m" in wl or "serving" in wl:
            H3 = run_sbert1m(args, dev, local, out, keep="serving" in wl)
            log("sbert1m done at %.0fs" % (time.time() - t0))
        if "serving" in wl and H3 is not None and not args.no_serve:
            run_serving(args, H2, H3, out)
            log("serving done at %.0fs" % (time.time() - t0))
        if H3 is not None:
            H3["ix"].close()
        H2["ix"].close()
        del H2, H3
        torch.cuda.empty_cache()
        if "deep1m" in wl:
            run_deep1m(args, dev, local, out)
            log("deep1m done at %.0fs" % (time.time() - t0))
        if "sift100k" in wl:
            run_sift100k(args, dev, local, out, threads)
            log("sift100k done at %.0fs" % (time.time() - t0))
    else:
        H2["ix"].close()
    if rank == 0:
        print(json.dumps(out))
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Reference arm: hnswlib (the reference's vendored copy) on the same graph
# ---------------------------------------------------------------------------
def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(local)
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    if not oracle.Hnsw.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhnswlib_ref.so not built"}))
        return 0
    x, q, g, gt, _ = sift10m_workload("cuda:%d" % local)
    efs, ks, _ = sift10m_params(len(q))
    h = oracle.Hnsw.from_graph(g.vectors, g.adjacency(), g.entry_point)
    n = args.ref_queries
    times = []
    for i in range(args.warmup + args.steps):
        s = (i * n) % len(q)
        t = time.time()
        lab, _ = h.search_mixed(q[s:s + n], ks[s:s + n], efs[s:s + n], threads)
        if i >= args.warmup:
            times.append(time.time() - t)
    lab, _ = h.search_mixed(q[:min(n, len(gt))], ks[:min(n, len(gt))], efs[:min(n, len(gt))], threads)
    rec = mixed_recall(lab, gt[:len(lab)], ks[:len(lab)])
    h.free()
    dt = sum(times)
    qps = n * len(times) / dt
    outj = {"metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / len(times) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded clipped-integer stand-in for SIFT10M)", "impl": "reference",
            "config": {"workload": WORKLOAD_SIFT10M, "queries_per_step": n, "recall": rec,
                       "step": "%d-query slice of the 100k mixed-parameter batch (the slice moves each step); "
                               "hnswlib searchKnn with each query's ef and k from the same medoid on the same "
                               "graph; mc has no hnswlib counterpart" % n,
                       "graph": "built by the same GPU builder as the GPU arm (data preparation, outside the timed "
                                "region)"},
            "cpu_baseline": {"kind": "reference", "cores": threads, "value": qps, "unit": "queries/s",
                             "isa": oracle.Hnsw.isa(), "cpu": oracle.Hnsw.cpu_model(),
                             "sample": "%d queries per step, hnswlib (the reference's vendored copy)" % n},
            "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(outj))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workloads", default="sift100k,deep1m,sbert1m,serving",
                    help="extra workloads after the sift10m headline (comma-separated; 'none' for the headline only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the continuous-batching measurements")
    ap.add_argument("--n-base", type=int, default=None, help="sift10m base size (scaled-down runs: checks only)")
    ap.add_argument("--n-queries", type=int, default=None)
    ap.add_argument("--deep1m-n", type=int, default=1_000_000)
    ap.add_argument("--sbert1m-n", type=int, default=1_000_000)
    ap.add_argument("--latency-samples", type=int, default=200)
    ap.add_argument("--ref-queries", type=int, default=4000, help="reference arm: queries per step")
    ap.add_argument("--graph-cache", default=None,
                    help="sift10m: load the graph and ground truth from this .npz if it exists, else save them "
                         "there (for repeated profiling runs of one workload)")
    ap.add_argument("--profile-region", action="store_true",
                    help="bracket only the timed headline steps with cudaProfilerStart/Stop and exit after them")
    ap.add_argument("--profile-throughput", action="store_true",
                    help="only deep1m 10k-query searches at the recall-0.95 throughput point, bracketed by "
                         "cudaProfilerStart/Stop (--steps searches after --warmup)")
    ap.add_argument("--profile-latency", action="store_true",
                    help="only deep1m batch-1 intra-query searches at the DST latency point, bracketed by "
                         "cudaProfilerStart/Stop (--steps searches after --warmup)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.n_base:
        SIFT10M["n"] = args.n_base
    SIFT10M["graph_cache"] = args.graph_cache
    if args.n_queries:
        SIFT10M["nq"] = args.n_queries
        SIFT10M["ngt"] = min(SIFT10M["ngt"], args.n_queries)
    from falcon_b200 import build as fb
    fb.build()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_latency:
        return profile_latency(args)
    if args.profile_throughput:
        return profile_throughput(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
