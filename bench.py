#!/usr/bin/env python
"""Benchmark of the B200 PDX search engine (one JSON line on rank 0).

Default workload (the headline metric's configuration): two-level IVF SQ8 search,
N = 1,000,000 unit-normalised float32 vectors, d = 1024, drawn from a 1,024-component Gaussian
mixture (sigma 0.25); 1,000 L1 / 32 L0 clusters; nprobe 32, k 20; batches of 10,000 queries
from the same mixture. A "step" is one search of one 10,000-query batch: normalization,
rotation, top-level (meso) search and the pruned PDX scan of 32 clusters per query.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--impl reference]

* value     -- queries/s with queries already in GPU memory (device-timed with CUDA events on
               the launching stream, the max over ranks for N > 1; N ranks each search their
               own batch against their own replica of the index: weak scaling).
* e2e       -- the same through the C ABI's host-buffer entry point (pdxg_search): pinned host
               queries in, host results out, copies inside the timed region.
* roofline  -- the search kernel alone: algorithmic bytes (index bytes the PDXearch algorithm
               reads, counted in-kernel) / its average event-timed duration, against the
               measured HBM copy bandwidth.
* cpu_baseline -- the reference's own search code (oracle/_ref, compiled from its headers) on
               this host's cores over a bounded sample of the same queries.
`--impl reference` times that reference CPU search as the benchmark's reference arm.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # headline: IVF2 SQ8 (two-level), exact per query
    "ivf2_sq8_1m_d1024": dict(itype="pdx_tree_u8", n=1_000_000, d=1024, comps=1024, sigma=0.25,
                              seed=2, unit=True, normalize=True, nlist=1000, nmeso=32, nprobe=32,
                              k=20, nq=10_000),
    # plain IVF F32 with ADSampling pruning
    "ivf_f32_100k_d128": dict(itype="pdx_f32", n=100_000, d=128, comps=256, sigma=0.3, seed=1,
                              unit=False, normalize=False, nlist=316, nmeso=0, nprobe=16, k=10,
                              nq=1_000),
    # exhaustive (all clusters in centroid order) F32, k = 100
    "flat_f32_2m_d768": dict(itype="pdx_f32", n=2_000_000, d=768, comps=2048, sigma=0.2, seed=3,
                             unit=True, normalize=True, nlist=5657, nmeso=0, nprobe=0, k=100,
                             nq=1024),
    # the same data, queries and tree shape with an F32 tree (PDXTreeIndex<F32>): the operating
    # point where recall@10 >= 0.95 is reachable (SQ8's quantisation caps recall at 0.911 here)
    "ivf2_f32_1m_d1024": dict(itype="pdx_tree_f32", n=1_000_000, d=1024, comps=1024, sigma=0.25,
                              seed=2, unit=True, normalize=True, nlist=1000, nmeso=32, nprobe=32,
                              k=20, nq=10_000),
    # precision form of the IVF2 SQ8 workload: BF16 tensor-core rotation and L1 centroid scores,
    # probe list widened by 10 %, FP32 rescore; 1,024-query batches over the same index
    "precision_ivf2_sq8_1m_d1024": dict(itype="pdx_tree_u8", n=1_000_000, d=1024, comps=1024,
                                        sigma=0.25, seed=2, unit=True, normalize=True, nlist=1000,
                                        nmeso=32, nprobe=32, k=20, nq=1024, probe_mode=1,
                                        dataset="ivf2_sq8_1m_d1024"),
}
DEFAULT_CONFIG = "ivf2_sq8_1m_d1024"
CACHE = os.environ.get("PDXG_BENCH_CACHE", os.path.join(tempfile.gettempdir(), "pdxg_bench"))
GT_QUERIES = 1000
RECALL_GATE = 0.95  # the headline metric's recall@10 operating point
L2_NOTE = "flushed between steps (256 MB write); index > L2"


def metric_name(config: str) -> str:
    return "QPS at recall@10>=0.95 (IVF2 SQ8 search)" if config == DEFAULT_CONFIG else f"QPS ({config})"


def workload_config(config: str, cfg: dict) -> dict:
    """The workload as both arms print it (identical keys and values in both)."""
    return {"workload": config, "index": cfg["itype"], "n": cfg["n"], "d": cfg["d"],
            "clusters": cfg["nlist"], "meso_clusters": cfg["nmeso"], "nprobe": cfg["nprobe"],
            "k": cfg["k"], "batch_queries": cfg["nq"], "l2": L2_NOTE}


def quality(rec10, rec_k, k, queries) -> dict:
    """Recall against the FP64 brute-force neighbours, and whether the metric's gate is met."""
    q = {"recall@10": None if rec10 is None else round(rec10, 4),
         f"recall@{k}": None if rec_k is None else round(rec_k, 4),
         "recall_gate": RECALL_GATE, "recall_gate_met": None if rec10 is None else bool(rec10 >= RECALL_GATE),
         "ground_truth": f"FP64 brute force, first {queries} queries of the batch"}
    return q


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------------------- data
def dataset(name: str, device: str):
    """Index file, query generator and ground truth, built once and cached on local disk."""
    from pdx_b200.builder import GaussianMixture, build_index
    cfg = CONFIGS[name]
    name = cfg.get("dataset", name)  # workloads over the same index share its files
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"{name}.pdx")
    gt_path = os.path.join(CACHE, f"{name}.gt.npy")
    gm = GaussianMixture(cfg["d"], cfg["comps"], cfg["sigma"], seed=cfg["seed"], unit_norm=cfg["unit"])
    if not (os.path.exists(path) and os.path.exists(gt_path)):
        t0 = time.time()
        X = gm.sample(cfg["n"], 0)
        f = build_index(X, cfg["itype"], num_clusters=cfg["nlist"], num_meso_clusters=cfg["nmeso"],
                        normalize=cfg["normalize"], seed=cfg["seed"], device=device)
        tmp = path + f".tmp{os.getpid()}"
        f.save(tmp)
        os.replace(tmp, path)
        del f
        Q = gm.sample(GT_QUERIES, 1)
        gt = ground_truth(X, Q, 100, device, cfg["normalize"])
        np.save(gt_path, gt)
        del X
        log(f"built {name} in {time.time() - t0:.1f}s -> {path} ({os.path.getsize(path) / 1e9:.2f} GB)")
    return path, gm, np.load(gt_path)


def run_build(name, cfg, device):
    """Native build (pdxg_build) of the workload's data from host memory to a loaded index,
    wall-clock with the device synchronized on both sides; recall@10 of the built index at the
    workload's nprobe next to the recall of the cached index the Python/torch builder made."""
    import torch
    from pdx_b200 import compiled
    from pdx_b200.builder import GaussianMixture
    gm = GaussianMixture(cfg["d"], cfg["comps"], cfg["sigma"], seed=cfg["seed"], unit_norm=cfg["unit"])
    X = gm.sample(cfg["n"], 0)
    Q = gm.sample(GT_QUERIES, 1)
    path, _, gt = dataset(name, device)
    times = []
    for rep in range(2):  # the first build also loads the module's kernels
        ix = compiled.PDXIndex(cfg["itype"], cfg["d"], seed=cfg["seed"], num_clusters=cfg["nlist"],
                               num_meso_clusters=cfg["nmeso"], normalize=cfg["normalize"],
                               device=torch.cuda.current_device())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ix.build_index(X)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    ix.set_nprobe(cfg["nprobe"])
    ids, _, cnt = ix.search_batch(Q, cfg["k"])
    rec = recall_at(ids, cnt, gt, 10)
    ref = compiled.load_index(path, device=torch.cuda.current_device())
    ref.set_nprobe(cfg["nprobe"])
    rids, _, rcnt = ref.search_batch(Q, cfg["k"])
    print(json.dumps({
        "metric": "index build time (native GPU build, host rows to loaded index)",
        "value": round(times[-1], 3), "unit": "s", "higher_is_better": False,
        "rows_per_s": round(cfg["n"] / times[-1]), "first_build_s": round(times[0], 3),
        "config": {"workload": cfg.get("dataset", name), "itype": cfg["itype"], "n": cfg["n"], "d": cfg["d"],
                   "nlist": cfg["nlist"], "nmeso": cfg["nmeso"], "kmeans_iters": 10},
        "recall@10": round(rec, 4), "recall@10_python_builder": round(recall_at(rids, rcnt, gt, 10), 4),
        "nprobe": cfg["nprobe"], "data": "synthetic"}), flush=True)


def run_maintenance(args, cfg, path, gm, device, n_ops=2000, n_ref_ops=200):
    """PDXTreeIndex::Append / Delete through the public API on the loaded workload index (host rows,
    wall clock per call, the device synchronized on both sides), then the device search of the
    workload's batch over the index with the tombstones left behind. The reference's own Append /
    Delete (oracle/_ref: its Cluster code, its rotation) run on the host beside it on a bounded
    sample. Rows are normalized on the host: a loaded index appends rows as given (LoadPDXIndex's
    default config does not normalize)."""
    import torch
    from pdx_b200 import compiled
    from pdx_b200.builder import normalize_rows
    if "tree" not in cfg["itype"]:
        raise SystemExit("--maintenance needs a tree workload")
    n = cfg["n"]
    rows = normalize_rows(gm.sample(n_ops, 21)) if cfg["normalize"] else gm.sample(n_ops, 21)
    victims = np.random.default_rng(5).choice(n, n_ops, replace=False)
    ix = compiled.load_index(path, device=torch.cuda.current_device())
    ix.set_nprobe(cfg["nprobe"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ix.append(n, rows[0])  # first call lays the clusters out at their capacity strides
    torch.cuda.synchronize()
    t_first = time.perf_counter() - t0
    t0 = time.perf_counter()
    for i in range(1, n_ops):
        ix.append(n + i, rows[i])
    torch.cuda.synchronize()
    t_app = time.perf_counter() - t0
    t0 = time.perf_counter()
    for v in victims:
        ix.delete(int(v))
    torch.cuda.synchronize()
    t_del = time.perf_counter() - t0
    # batched appends (one rotation and top-level search per 4,096 rows)
    n_batch = 50_000
    brows = normalize_rows(gm.sample(n_batch, 22)) if cfg["normalize"] else gm.sample(n_batch, 22)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for a in range(0, n_batch, 4096):
        ix.append_batch(n + n_ops + a, brows[a:a + 4096])
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    st = ix.maintenance_stats()
    # search with tombstones (the scan's tombstone-masking instantiation)
    nq, k = cfg["nq"], cfg["k"]
    q = torch.from_numpy(gm.sample(nq, 1)).to(device)
    ids = torch.empty((nq, k), dtype=torch.int32, device=device)
    ds = torch.empty((nq, k), dtype=torch.float32, device=device)
    cnt = torch.empty(nq, dtype=torch.int32, device=device)
    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    for _ in range(3):
        ix.search_device(q.data_ptr(), nq, k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(), stream=sp)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    reps = 10
    for _ in range(reps):
        ix.search_device(q.data_ptr(), nq, k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(), stream=sp)
    b.record(stream)
    torch.cuda.synchronize()
    qps = nq * reps / (a.elapsed_time(b) / 1e3)
    deleted = set(int(v) for v in victims)
    found_deleted = int(np.isin(ids.cpu().numpy().view(np.uint32), list(deleted)).sum())
    ref_line = None
    try:
        from oracle.oracle import Reference
        if Reference.available():
            ref = Reference(path)
            t0 = time.perf_counter()
            for i in range(n_ref_ops):
                ref.append(n + i, rows[i])
            r_app = time.perf_counter() - t0
            t0 = time.perf_counter()
            for v in victims[:n_ref_ops]:
                ref.delete(int(v))
            r_del = time.perf_counter() - t0
            ref.close()
            ref_line = {"appends_per_s": round(n_ref_ops / r_app, 1), "deletes_per_s": round(n_ref_ops / r_del, 1),
                        "cores": 1, "kind": "reference", "sample": f"first {n_ref_ops} appends and deletes"}
    except Exception as e:  # the CPU baseline is reported, never required
        ref_line = {"unavailable": str(e)[:200]}
    print(json.dumps({
        "metric": "Append / Delete throughput on the loaded tree index (host rows, one call each)",
        "value": round((n_ops - 1) / t_app, 1), "unit": "appends/s", "higher_is_better": True,
        "deletes_per_s": round(n_ops / t_del, 1), "first_append_s": round(t_first, 3),
        "batch_appends_per_s": round(n_batch / t_batch, 1), "batch_rows": 4096,
        "maintenance_stats": st,
        "search_after": {"qps_device": round(qps, 1), "batch_queries": nq, "nprobe": cfg["nprobe"], "k": k,
                         "deleted_rows_returned": found_deleted},
        "config": {"workload": cfg.get("dataset", args.config), "index": cfg["itype"], "n": n, "d": cfg["d"],
                   "ops": n_ops},
        "cpu_baseline": ref_line, "data": "synthetic"}), flush=True)


def ground_truth(X, Q, k, device, normalize):
    """Exact FP64 L2 neighbours in the original (normalized when the index is) space."""
    import torch
    from pdx_b200.builder import normalize_rows
    if normalize:
        Q = normalize_rows(Q)
    q = torch.from_numpy(Q).to(device).double()
    best_d = torch.full((len(Q), k), float("inf"), dtype=torch.float64, device=device)
    best_i = torch.zeros((len(Q), k), dtype=torch.int64, device=device)
    step = 1 << 17
    for s in range(0, X.shape[0], step):
        xs = X[s:s + step]
        if normalize:
            xs = normalize_rows(xs)
        x = torch.from_numpy(xs).to(device).double()
        d2 = (q * q).sum(1, keepdim=True) - 2.0 * q @ x.T + (x * x).sum(1)[None, :]
        cd = torch.cat([best_d, d2], 1)
        ci = torch.cat([best_i, torch.arange(s, s + len(xs), device=device)[None, :].expand(len(Q), -1)], 1)
        best_d, idx = torch.topk(cd, k, dim=1, largest=False)
        best_i = torch.gather(ci, 1, idx)
    return best_i.cpu().numpy().astype(np.int64)


def unique_bytes(ix, nq, nprobe, elem):
    """Index bytes one batch must read at least once, from the visit orders of the last device
    search (computed ahead of the scan): the full vectors of every cluster that is some query's
    Start cluster (its first non-empty visited cluster), and the first warmup checkpoint's
    vertical rows (min(16, d_v) dims) of every cluster visited after a Start. Counted once per
    batch however many queries read them."""
    orders, counts = ix.last_visit_orders(nq, nprobe)
    n1 = ix.get_num_clusters()
    size = np.array([ix.get_cluster_size(c) for c in range(n1)], np.int64)
    d = ix.get_num_dimensions()
    first = np.zeros(n1, bool)
    later = np.zeros(n1, bool)
    visits = 0
    for i in range(nq):
        o = orders[i, :counts[i]]
        o = o[size[o] > 0]
        if len(o):
            first[o[0]] = True
            later[o[1:]] = True
            visits += len(o)
    cp1 = min(16, d)
    return {"start_rows": int(size[first].sum()) * d * elem,
            "first_checkpoint_rows": int(size[later].sum()) * cp1 * elem,
            "clusters_started": int(first.sum()), "clusters_visited_later": int(later.sum()),
            "visits": visits}


def recall_at(ids, counts, gt, k):
    hits = 0
    for i in range(len(gt)):
        hits += len(set(ids[i, :min(k, counts[i])].tolist()) & set(gt[i, :k].tolist()))
    return hits / (k * len(gt))


# ----------------------------------------------------------------------------- ranks
def max_over_ranks(x: float, device) -> float:
    """The slowest rank's figure (1 process: x itself)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_qps(queries_per_rank: int, steps: int, world: int, max_ms: float) -> float:
    """All ranks' queries over the slowest rank's time (replicas: weak scaling)."""
    return world * queries_per_rank * steps / (max_ms / 1e3)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, gpu_index: int):
        self.path = os.path.join(tempfile.gettempdir(), f"pdxg_clocks_{os.getpid()}.csv")
        fields = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                  "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={fields}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- CPU reference
def reference_lib_flavour():
    from oracle.oracle import Reference, cpu_has_avx512_vnni
    if cpu_has_avx512_vnni() and Reference.available("avx512"):
        return "avx512"
    return "avx2"


def time_reference(path, queries, cfg, threads, budget_s=12.0, max_queries=None):
    """QPS of the reference's own search over a bounded sample, all `threads` host threads."""
    from oracle.oracle import Reference
    flav = reference_lib_flavour()
    ref = Reference(path, flav)
    ref.set_nprobe(cfg["nprobe"])
    k = cfg["k"]
    probe_n = min(len(queries), max(threads * 2, 32))
    t0 = time.perf_counter()
    ref.search_batch(queries[:probe_n], k, n_threads=threads)
    per_q = (time.perf_counter() - t0) / probe_n
    n = int(min(len(queries), max(probe_n, budget_s / max(per_q, 1e-9))))
    if max_queries:
        n = min(n, max_queries)
    t0 = time.perf_counter()
    ids, ds, cnt = ref.search_batch(queries[:n], k, n_threads=threads)
    dt = time.perf_counter() - t0
    ref.close()
    return n / dt, n, dt, flav, (ids, cnt)


# ----------------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--config", default=DEFAULT_CONFIG, choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--threads", type=int, default=0, help="threads per query CTA (0 = auto)")
    ap.add_argument("--top-mode", type=int, default=None,
                    help="tree top level: 0 auto, 1 per query, 2 batched warp-per-query kernel")
    ap.add_argument("--rotation-mode", type=int, default=None,
                    help="0: tcgen05 TF32x3 rotation when available (default), 1: FP32 SIMT GEMM")
    ap.add_argument("--probe-mode", type=int, default=None,
                    help="0 reference probe, 1 BF16 tensor-core probe, 2 FP8-E4M3 centroid scores")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the engine's default forms")
    ap.add_argument("--no-graph", action="store_true", help="launch each step directly, not from a CUDA graph")
    ap.add_argument("--nprobe", type=int, default=None, help="override the workload's nprobe")
    ap.add_argument("--nq", type=int, default=None, help="override the workload's batch size")
    ap.add_argument("--scan-mode", type=int, default=None,
                    help="U8 scan after a batched Start: 0 cluster-major (default), 1 per-query kernel")
    ap.add_argument("--profile", action="store_true",
                    help="run only the warm-up and timed search steps (for ncu captures); no bench line")
    ap.add_argument("--sweep", action="store_true",
                    help="print recall@10 / QPS over an nprobe ladder and exit")
    ap.add_argument("--serve", action="store_true",
                    help="serving mix over the index: Poisson arrivals, mixed k / nprobe / filters")
    ap.add_argument("--serve-rates", default="5000,20000,50000,100000,200000",
                    help="arrival rates (requests/s) of the serving run")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="arrivals per rate (seconds)")
    ap.add_argument("--build", action="store_true",
                    help="time the native GPU index build of the workload's data and exit")
    ap.add_argument("--maintenance", action="store_true",
                    help="time Append / Delete on the workload's tree index, then search with tombstones")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    cfg = dict(CONFIGS[args.config])
    if args.nprobe is not None:
        cfg["nprobe"] = args.nprobe
    if args.nq is not None:
        cfg["nq"] = args.nq

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    device = f"cuda:{local_rank}"
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(minutes=10))

    def barrier():
        if world > 1:
            dist.barrier()

    if args.build:
        if rank == 0:
            run_build(args.config, cfg, device)
        if world > 1:
            dist.destroy_process_group()
        return

    # the index is built once (rank 0) into a local cache shared by the ranks
    if rank == 0:
        path, gm, gt = dataset(args.config, device)
    barrier()
    if rank != 0:
        path, gm, gt = dataset(args.config, device)

    if args.impl == "reference":
        run_reference_arm(args, cfg, path, gm, gt, rank, world)
        if world > 1:
            dist.destroy_process_group()
        return

    if args.maintenance:
        if rank == 0:
            run_maintenance(args, cfg, path, gm, device)
        if world > 1:
            dist.destroy_process_group()
        return

    if args.serve:
        run_serve(args, cfg, path, gm, gt, rank, world, local_rank)
        if world > 1:
            dist.destroy_process_group()
        return

    from pdx_b200 import compiled
    ix = compiled.load_index(path, device=local_rank)
    ix.set_nprobe(cfg["nprobe"])
    if args.threads:
        ix.set_threads_per_query(args.threads)
    if args.top_mode is not None:
        ix.set_top_level_mode(args.top_mode)
    if args.rotation_mode is not None:
        ix.set_rotation_mode(args.rotation_mode)
    if args.scan_mode is not None:
        ix.set_scan_mode(args.scan_mode)
    probe_mode = cfg.get("probe_mode", 0) if args.probe_mode is None else args.probe_mode
    if probe_mode:
        ix.set_probe_mode(probe_mode)
    rot_tc = ix.rotation_uses_tensor_cores()
    nq, k, d = cfg["nq"], cfg["k"], cfg["d"]
    Qh = gm.sample(nq, 1 + rank)  # rank-specific batch; the first GT_QUERIES match the GT
    # a dedicated stream: the events below and the engine's launches must share it (handle 0,
    # the legacy default stream, would select the index's own stream instead)
    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    q_dev = torch.from_numpy(Qh).to(device)
    ids_dev = torch.empty((nq, k), dtype=torch.int32, device=device)
    dist_dev = torch.empty((nq, k), dtype=torch.float32, device=device)
    cnt_dev = torch.empty(nq, dtype=torch.int32, device=device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)  # > 126 MB L2

    tuned = None
    if not args.no_autotune and not args.sweep and args.threads == 0 and args.top_mode is None:
        tuned = ix.autotune(q_dev.data_ptr(), nq, k)
    graph = None
    if not args.no_graph and not args.sweep:
        graph = ix.capture(q_dev.data_ptr(), nq, k, ids_dev.data_ptr(), dist_dev.data_ptr(), cnt_dev.data_ptr())

    def step():
        if graph is not None:
            graph.launch(sp)
        else:
            ix.search_device(q_dev.data_ptr(), nq, k, ids_dev.data_ptr(), dist_dev.data_ptr(),
                             cnt_dev.data_ptr(), stream=sp)

    if args.profile:
        for _ in range(args.warmup + args.steps):
            step()
            flush.zero_()
        torch.cuda.synchronize()
        log(f"profile run: {args.warmup + args.steps} steps of {nq} queries, {ix.last_launch_count()} engine "
            f"launches per step")
        if world > 1:
            dist.destroy_process_group()
        return
    if args.sweep:
        gq = torch.from_numpy(Qh[:len(gt)]).to(device)
        for npb in (16, 24, 32, 40, 48, 64, 80, 96, 128, 192, 256):
            ix.set_nprobe(npb)
            ix.search_device(gq.data_ptr(), len(gt), k, ids_dev.data_ptr(), dist_dev.data_ptr(),
                             cnt_dev.data_ptr(), stream=sp)
            torch.cuda.synchronize()
            ids_np = ids_dev[:len(gt)].cpu().numpy().view(np.uint32)
            cnt_np = cnt_dev[:len(gt)].cpu().numpy().view(np.uint32)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            torch.cuda.synchronize()
            print(json.dumps({"nprobe": npb, "recall@10": round(recall_at(ids_np, cnt_np, gt, 10), 4),
                              f"recall@{k}": round(recall_at(ids_np, cnt_np, gt, k), 4),
                              "qps": round(nq / (a.elapsed_time(b) / 1e3), 1)}), flush=True)
        return
    for _ in range(args.warmup):
        step()
        flush.zero_()
    torch.cuda.synchronize()
    if graph is not None:  # the graph replays the launches of its capture run
        ix.search_device(q_dev.data_ptr(), nq, k, ids_dev.data_ptr(), dist_dev.data_ptr(),
                         cnt_dev.data_ptr(), stream=sp)
        torch.cuda.synchronize()
    launches_per_step = ix.last_launch_count()
    # quality of this batch's results (rank 0's batch carries the ground-truth queries)
    ids_np = ids_dev.cpu().numpy().view(np.uint32)
    cnt_np = cnt_dev.cpu().numpy().view(np.uint32)
    rec10 = recall_at(ids_np, cnt_np, gt, 10) if rank == 0 else None
    rec_k = recall_at(ids_np, cnt_np, gt, k) if rank == 0 else None

    # ---- timed region: K steps, per-step CUDA events, L2 flushed between steps (untimed)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        starts[i].record(stream)
        step()
        ends[i].record(stream)
        flush.zero_()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = max_over_ranks(sum(step_ms), device)
    value = whole_job_qps(nq, args.steps, world, total_ms)

    # ---- roofline of the search kernel alone (prepared queries, same batch)
    prepared = torch.from_numpy(ix.prepare_queries(Qh)).to(device)
    ix.search_device(prepared.data_ptr(), nq, k, ids_dev.data_ptr(), dist_dev.data_ptr(),
                     cnt_dev.data_ptr(), stream=sp, transformed=True, stats=True)
    stats = ix.last_stats()
    scan_stats = ix.last_scan_stats()
    # the scan kernel alone: events the engine records around its own launches on `stream`
    times = []
    for i in range(args.steps):
        ix.search_device(q_dev.data_ptr(), nq, k, ids_dev.data_ptr(), dist_dev.data_ptr(),
                         cnt_dev.data_ptr(), stream=sp, time_kernels=True)
        times.append(ix.kernel_times())
        flush.zero_()
    torch.cuda.synchronize()
    kernels_ms = {key: round(statistics.mean(t[key] for t in times), 4) for key in times[0]}
    kern_ms = statistics.mean(t["search_kernel"] for t in times)
    start_ms = statistics.mean(t["start"] for t in times)
    top_ms = statistics.mean(t["top_level"] for t in times)
    prep_ms = statistics.mean(t["prepare"] for t in times)
    bp = stats["bytes_by_phase"]
    batched_start = start_ms > 0.0
    # index bytes the scan kernel itself reads per the algorithm: warmup rows, survivor rows,
    # centroids of an in-kernel probe, and for each query's first cluster either its full
    # vectors (Start in the kernel) or the 4-byte distances the batched Start wrote for it
    start_reads = (bp["start"] // d) * 4 if batched_start else bp["start"]
    scan_bytes = bp["warmup"] + bp["survivor_horizontal"] + bp["survivor_vertical"] + bp["probe"] + start_reads
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = float(json.load(open(peaks_path))["hbm_gbs"])
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = scan_bytes / (kern_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(args.config)

    # ---- probe-set error against the FP64 nearest L1 centroids (probe modes 1 and 2)
    probe = None
    if probe_mode and rank == 0:
        probe = probe_report(ix, path, Qh[:len(gt)], cfg, k, gt, device, sp, probe_mode)

    # ---- plain path: one query per launch (p50 / p99 latency)
    lat = []
    n_plain = min(300, nq)
    for i in range(n_plain + 10):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ix.search_device(q_dev[i].data_ptr(), 1, k, ids_dev.data_ptr(), dist_dev.data_ptr(),
                         cnt_dev.data_ptr(), stream=sp)
        b.record(stream)
        b.synchronize()
        if i >= 10:
            lat.append(a.elapsed_time(b))
    plain_qps = 1e3 / statistics.mean(lat)

    # ---- end to end through the C ABI with host buffers (pinned), copies inside the region
    q_pin = torch.from_numpy(Qh).pin_memory()
    ids_pin = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    d_pin = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    c_pin = torch.empty(nq, dtype=torch.int32).pin_memory()
    lib = compiled.library()
    import ctypes as C

    def e2e_step():
        rc = lib.pdxg_search(ix.handle.ptr, C.c_void_p(q_pin.data_ptr()), nq, k, 0,
                             C.c_void_p(ids_pin.data_ptr()), C.c_void_p(d_pin.data_ptr()),
                             C.c_void_p(c_pin.data_ptr()))
        if rc != 0:
            raise RuntimeError(lib.pdxg_last_error().decode())

    for _ in range(2):
        e2e_step()
    e2e_times = []
    for _ in range(max(3, args.steps // 2)):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.mean(e2e_times), device)
    e2e_value = whole_job_qps(nq, 1, world, e2e_s * 1e3)
    # the query upload alone (pinned host -> device, the same bytes), to explain e2e vs value
    h2d_ms = []
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        q_dev.copy_(q_pin, non_blocking=True)
        b.record(stream)
        b.synchronize()
        h2d_ms.append(a.elapsed_time(b))
    h2d_gbs = nq * d * 4 / (min(h2d_ms) * 1e-3) / 1e9

    # ---- CPU baseline: the reference's own search on this host, bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            qps, n, dt, flav, _ = time_reference(path, Qh, cfg, threads)
            cpu = {"value": round(qps, 1), "unit": "queries/s", "cores": threads, "kind": "reference",
                   "sample": f"{n} of the {nq} bench queries, {dt:.1f}s, reference PDXearch built from "
                             f"its headers ({flav}), one searcher pair per thread"}
        except Exception as e:  # the baseline must not sink the GPU measurement
            cpu = {"value": None, "unit": "queries/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": metric_name(args.config),
            "value": round(value, 1),
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u8" if "u8" in cfg["itype"] else "f32",
            "data": "synthetic (seeded Gaussian mixture; no public dataset in the container)",
            "config": workload_config(args.config, cfg),
            "quality": quality(rec10, rec_k, k, len(gt)),
            "details": {
                "plain_one_query_per_launch_qps": round(plain_qps, 1),
                "batched_over_plain": round(value / world / plain_qps, 1),
                "latency_ms_plain": {"p50": round(float(np.percentile(lat, 50)), 3),
                                     "p99": round(float(np.percentile(lat, 99)), 3)},
                "latency_ms_batch": {"p50": round(float(np.percentile(step_ms, 50)), 3),
                                     "p99": round(float(np.percentile(step_ms, 99)), 3)},
                "parallelism": f"replicas{world}" if world > 1 else "single",
                "rotation": ("tcgen05 BF16" if probe_mode else ("tcgen05 TF32x3" if rot_tc else "FP32 SIMT")),
                "probe": probe if probe_mode else "reference (exact)",
                "autotuned": tuned if tuned else "off",
                "step_launch": "CUDA graph" if graph is not None else "direct",
            },
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": "search_kernel", "kernel_ms": round(kern_ms, 3),
                         "algorithmic_bytes_per_launch": scan_bytes, "peak_source": peak_src,
                         "other_kernels_ms": {("precision probe (rotation + scores + select)" if probe_mode
                                               else "tree top level"): round(top_ms, 3),
                                              "batched start": round(start_ms, 3),
                                              "query preparation": round(prep_ms, 3)},
                         "batched_start_replaces_bytes": bp["start"] if batched_start else 0,
                         "top_level_bytes_l2_resident": bp["top_level"],
                         "clusters_visited": stats["clusters_visited"],
                         "kernels_ms": kernels_ms,
                         "scan_counters": scan_stats,
                         "bytes_by_phase": stats["bytes_by_phase"],
                         "cycles_by_phase": stats["cycles_by_phase"]},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 1), "unit": "queries/s",
                    "h2d_bytes_per_step": nq * d * 4,
                    "d2h_bytes_per_step": nq * k * 8 + nq * 4,
                    "h2d_gbs_measured": round(h2d_gbs, 1),
                    "h2d_ms_per_step": round(min(h2d_ms), 3)},
            # per step: query preparation + [tree top level] + scan, as counted by the engine
            "gpu_launches": args.steps * launches_per_step,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def probe_report(ix, path, Q, cfg, k, gt, device, stream, restore_mode):
    """Probe-set mismatch of the reduced-precision probe against the FP64 nearest L1 centroids
    of the FP64-normalized, FP64-rotated queries, and recall of its results; for probe modes 1
    (BF16 scores) and 2 (FP8-E4M3 scores). Leaves the index in its original probe mode."""
    import torch
    from pdx_b200.layout import read_index
    f = read_index(open(path, "rb").read())
    rot = np.asarray(f.rotation, np.float64)
    if f.l0 is not None:  # tree: the L1 centroids are the meso clusters' vectors
        C = np.zeros((f.l1.nclusters, f.d), np.float64)
        for emb, ids in zip(f.l0.embeddings, f.l0.row_ids):
            C[ids] = emb
    else:
        C = np.asarray(f.l1.centroids, np.float64)
    Qd = Q.astype(np.float64)
    if cfg["normalize"]:
        Qd = Qd / np.linalg.norm(Qd, axis=1, keepdims=True)
    R = torch.from_numpy(Qd @ rot).to(device)
    Ct = torch.from_numpy(C).to(device)
    nprobe = cfg["nprobe"]
    d2 = (R * R).sum(1, keepdim=True) - 2.0 * R @ Ct.T + (Ct * Ct).sum(1)[None, :]
    truth = torch.topk(d2, nprobe, dim=1, largest=False).indices.cpu().numpy()
    nq = len(Q)
    q = torch.from_numpy(np.ascontiguousarray(Q)).to(device)
    ids = torch.empty((nq, k), dtype=torch.int32, device=device)
    ds = torch.empty((nq, k), dtype=torch.float32, device=device)
    cnt = torch.empty(nq, dtype=torch.int32, device=device)
    out = {"vs": "FP64 nearest L1 centroids", "queries": nq, "widened_list": "ceil(1.1 nprobe)"}
    for mode, name in ((0, "reference_probe"), (1, "bf16"), (2, "fp8_e4m3")):
        if mode == 0 and f.l0 is None:
            continue  # the flat reference probe runs inside the scan kernel: no visit orders
        ix.set_probe_mode(mode)
        ix.search_device(q.data_ptr(), nq, k, ids.data_ptr(), ds.data_ptr(), cnt.data_ptr(), stream=stream)
        torch.cuda.synchronize()
        orders, counts = ix.last_visit_orders(nq, nprobe)
        miss = 1.0 - float(np.mean([len(set(orders[i, :counts[i]].tolist()) & set(truth[i].tolist())) / nprobe
                                    for i in range(nq)]))
        ids_np = ids.cpu().numpy().view(np.uint32)
        cnt_np = cnt.cpu().numpy().view(np.uint32)
        out[name] = {"probe_set_mismatch": round(miss, 5), "recall@10": round(recall_at(ids_np, cnt_np, gt, 10), 4),
                     f"recall@{k}": round(recall_at(ids_np, cnt_np, gt, k), 4)}
    ix.set_probe_mode(restore_mode)
    return out


def run_serve(args, cfg, path, gm, gt, rank, world, local_rank):
    """Serving mix over the index: Poisson arrivals at each rate of the ladder, k uniform in
    {10, 20, 100}, nprobe uniform in {8, 32, 64}, half of the requests carrying one of 64
    registered row-id filters of log-uniform selectivity in [0.001, 0.5]; continuous batching
    over 3 contexts. Reports achieved QPS and p50 / p99 latency per rate, and the saturated QPS
    (all requests queued at once) as the value."""
    import torch
    from pdx_b200 import compiled
    from pdx_b200.serving import Server, make_filters, poisson_mix
    ix = compiled.load_index(path, device=local_rank)
    filters = make_filters(ix, 64, seed=5)
    srv = Server(ix, max_batch=4096, n_contexts=3, k_max=100)
    rates = [float(r) for r in args.serve_rates.split(",") if r]
    nmax = 200_000
    Qall = gm.sample(nmax, 1 + rank)  # the first GT_QUERIES match the ground truth
    # warm-up (allocations, module load) at saturation
    srv.run(poisson_mix(Qall[:20_000], 0.0, filters, seed=4), realtime=False)
    torch.cuda.synchronize()
    ladder = []
    sampler = ClockSampler(local_rank)
    for rate in rates:
        n = int(min(nmax, max(2000, rate * args.serve_seconds)))
        w = poisson_mix(Qall[:n], rate, filters, seed=5)
        out = srv.run(w, realtime=True)
        ladder.append({"rate": rate, "requests": n, "qps": round(n / out.wall, 1),
                       "p50_ms": round(float(np.percentile(out.latency, 50)) * 1e3, 3),
                       "p99_ms": round(float(np.percentile(out.latency, 99)) * 1e3, 3),
                       "batches": int(out.batch.max()) + 1})
        log(f"serve rate {rate:.0f}/s: {ladder[-1]}")
    w = poisson_mix(Qall, 0.0, filters, seed=5)
    t_sat = []
    for _ in range(max(1, args.steps // 10)):
        out = srv.run(w, realtime=False)
        t_sat.append(out.wall)
    clocks = sampler.stop()
    sat_qps = nmax / min(t_sat)
    # recall@10 of the unfiltered requests that have ground truth
    g = min(len(gt), nmax)
    plain = np.nonzero(w.filter_id[:g] < 0)[0]
    hits = 0
    for i in plain:
        ids_i, _ = out.result(i)
        hits += len(set(ids_i[:10].tolist()) & set(gt[i, :10].tolist()))
    rec10 = hits / (10 * max(1, len(plain)))
    srv.close()
    if rank == 0:
        print(json.dumps({
            "metric": "served QPS (serving mix over the IVF2 SQ8 index)", "value": round(sat_qps, 1),
            "unit": "queries/s", "n_gpus": world, "steps": len(t_sat), "warmup": 1,
            "ms_per_step": round(1e3 * min(t_sat), 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded Gaussian mixture)",
            "config": {"workload": f"serve_{args.config}", "requests_saturated": nmax,
                       "k": [10, 20, 100], "nprobe": [8, 32, 64], "filtered_share": 0.5,
                       "filters": "64 registered, selectivity log-uniform [0.001, 0.5]",
                       "contexts": 3, "max_batch": 4096, "recall@10_unfiltered": round(rec10, 4),
                       "ladder": ladder},
            "clocks": clocks}), flush=True)


def u8_wrap_record(path, Q, cfg, flav, ids, ds, cnt, threads, sample=500):
    """Whether the AVX512-VNNI build of the reference's U8 distance can wrap on this workload.

    That build accumulates vpdpbusds(acc, |q - x|, |q - x|) with the second operand read as
    signed bytes (avx512_computers.hpp:156), so a per-dimension |q - x| >= 128 gives a wrong
    sum; the AVX2 and scalar builds are exact. Recorded: the largest |q - x| any quantized query
    dimension of the batch can reach against any stored vector (from per-dimension min / max,
    an upper bound), and whether the timed build's results equal the exact AVX2 build's on a
    sample of the queries. The bound covers the batch's first 1,000 queries."""
    from oracle.oracle import Port, Reference
    from pdx_b200.layout import read_index
    f = read_index(open(path, "rb").read())
    lo = np.full(f.d, 255, np.int32)
    hi = np.zeros(f.d, np.int32)
    for emb in f.l1.embeddings:
        if len(emb):
            e = np.asarray(emb, np.int32)
            lo = np.minimum(lo, e.min(0))
            hi = np.maximum(hi, e.max(0))
    port = Port(path)
    qmin = np.full(f.d, 255, np.int32)
    qmax = np.zeros(f.d, np.int32)
    for q in Q[:1000]:
        qq = port.quantize(port.prepare_query(q)).astype(np.int32)
        qmin = np.minimum(qmin, qq)
        qmax = np.maximum(qmax, qq)
    port.close()
    bound = int(max((qmax - lo).max(), (hi - qmin).max()))
    out = {"max_abs_q_minus_x_bound": bound, "wrap_possible": bound >= 128, "timed_build": flav}
    if flav != "avx2":
        n = min(sample, len(ids))
        exact = Reference(path, "avx2")
        exact.set_nprobe(cfg["nprobe"])
        eids, eds, ecnt = exact.search_batch(Q[:n], cfg["k"], n_threads=threads)
        exact.close()
        same = all(np.array_equal(eds[i, :ecnt[i]], ds[i, :cnt[i]]) and
                   set(eids[i, :ecnt[i]].tolist()) == set(ids[i, :cnt[i]].tolist()) for i in range(n))
        out["timed_equals_avx2_on_sample"] = bool(same)
        out["sample_queries"] = n
    return out


def run_reference_arm(args, cfg, path, gm, gt, rank, world):
    if rank != 0:
        return
    nq, k = cfg["nq"], cfg["k"]
    Qh = gm.sample(nq, 1)
    threads = os.cpu_count() or 1
    # size each step so that warmup + steps stay within a few minutes
    qps0, n0, dt0, flav, _ = time_reference(path, Qh, cfg, threads, budget_s=4.0)
    per_step = int(max(threads, min(nq, qps0 * 150.0 / max(1, args.steps + args.warmup))))
    from oracle.oracle import Reference
    ref = Reference(path, flav)
    ref.set_nprobe(cfg["nprobe"])
    for i in range(args.warmup):
        ref.search_batch(Qh[:per_step], k, n_threads=threads)
    times = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        ids, ds, cnt = ref.search_batch(Qh[:per_step], k, n_threads=threads)
        times.append(time.perf_counter() - t0)
    ng = min(per_step, len(gt))
    rec10 = recall_at(ids[:ng], cnt, gt[:ng], 10)
    rec_k = recall_at(ids[:ng], cnt, gt[:ng], k)
    ref.close()
    wrap = u8_wrap_record(path, Qh, cfg, flav, ids, ds, cnt, threads) if "u8" in cfg["itype"] else None
    total = sum(times)
    value = per_step * args.steps / total
    line = {
        "impl": "reference",
        "metric": metric_name(args.config),
        "value": round(value, 1), "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8" if "u8" in cfg["itype"] else "f32",
        "data": "synthetic (seeded Gaussian mixture; no public dataset in the container)",
        "config": workload_config(args.config, cfg),
        "quality": quality(rec10, rec_k, k, ng),
        "details": {"queries_per_step": per_step, "u8_wrap": wrap},
        "cpu_baseline": {"value": round(value, 1), "unit": "queries/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{per_step} queries per step of the {nq}-query batch ({flav} build)"},
        "e2e": {"value": round(value, 1), "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
