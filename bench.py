#!/usr/bin/env python
"""Benchmark: exact-result range queries/s on the batched configuration, one B200 per rank.

Workload (default --config batched): RandomKmeans-style index N=10,000,000, D=8, height 4, ratios
100,50,20, sigma divisor 3.0, seed 1 (generated in memory, byte-identical to the reference's
--gen-index); 4096 range boxes centred on uniformly chosen data points with per-dimension
half-widths log-uniform in [0.1%, 10%] of the extent. A step is one batched exact traversal of all
4096 boxes (all levels, the exact final filter and the per-query result offsets).

Reported on one JSON line (rank 0):
  value           whole-job exact queries/s with the boxes resident in HBM (device events)
  e2e             the same through the public host-buffer API (boxes H2D from pinned memory,
                  offsets + ids D2H, every step inside the timed region)
  plain           one query at a time through the same engine (the >=5x denominator)
  roofline        the dominant level (longest event time): its algorithmic bytes / its duration,
                  with every level's bytes and rate
  cpu_baseline    the CPU port of the traversal (oracle) on all host cores, bounded sample
Multi-GPU: replicas only (the path needs no exchange); every rank runs its own batches and the
time is the max over ranks.
"""
import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))


def _package():
    pkg_dir = os.path.join(REPO, "t-blaeq_b200")
    spec = importlib.util.spec_from_file_location("tblaeq_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tblaeq_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _workloads():
    """t-blaeq_b200/workloads.py on its own (it needs numpy only), without the package around it."""
    spec = importlib.util.spec_from_file_location("tblaeq_workloads", os.path.join(REPO, "t-blaeq_b200",
                                                                                   "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "20"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to start: wait for its first sample, so that a timed region
            # of a fraction of a second is sampled throughout.
            t0 = time.perf_counter()
            while not self.lines and self.proc.poll() is None and time.perf_counter() - t0 < 5.0:
                time.sleep(0.005)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
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
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def oracle_index_from_handler(oracle, h):
    info = h.info()
    L = info["intervals"]
    D = info["D"]
    col_res = [h.host_array(1, l) for l in range(L)]
    pvals = [h.host_array(0, l).reshape(-1, D) for l in range(L)]
    radius = [h.host_array(2, l) for l in range(L)]
    maps = [None] + [h.host_array(3, m) for m in range(1, info["height"])]
    cids = h.host_array(4)
    cvals = h.host_array(5).reshape(-1, D)
    return oracle.OracleIndex(D, info["N"], info["height"], info["ratios"], info["meshSizes"], col_res,
                              [np.diff(c) for c in col_res], [np.arange(len(p), dtype=np.uint64) for p in pvals],
                              pvals, radius, maps, cids, cvals)


def max_over_ranks(value: float) -> float:
    """The largest of every rank's value (1 rank: the value itself). Replicas are timed on their own
    device and the job takes as long as its slowest rank; NCCL reduces on the GPU, other backends
    on the host."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    import torch
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job throughput: every replica processed units_per_rank in at most seconds_max."""
    return units_per_rank * world / seconds_max


def profiled_traffic(cfg_name, nq, level, height):
    """DRAM bytes (read + write) of one launch of `level` at this exact workload, from the committed
    ncu summary (`traffic_bytes_per_launch_level<m>:` lines; one capture of the same command; ncu
    is never run by the benchmark)."""
    if cfg_name != "batched" or nq != 4096:
        return None
    path = os.path.join(REPO, "profiles", "expand_batched_range_n10m_d8.md")
    if not os.path.exists(path):
        return None
    import re
    m = re.search(r"^traffic_bytes_per_launch_level" + str(level) + r":\s*(\d+)", open(path).read(), re.M)
    return int(m.group(1)) if m else None


def cpu_port_qps(oracle, oidx, sub, Q, budget_s=20.0, min_q=32):
    """Time the CPU port of the exact traversal on all host cores over a bounded sample."""
    threads = os.cpu_count() or 1
    n = min_q
    done, elapsed = 0, 0.0
    while elapsed < budget_s and done < len(Q):
        batch = Q[done:done + n]
        t0 = time.perf_counter()
        oracle.exact_query(oidx, oracle.RANGE, batch, sub=sub, threads=threads)
        dt = time.perf_counter() - t0
        done += len(batch)
        elapsed += dt
        n = min(len(Q) - done, max(n, int(len(batch) * max(1.0, (budget_s - elapsed) / max(dt, 1e-6) / 2))))
        if n <= 0:
            break
    return done / elapsed, threads, done


class OracleWorkloadView:
    """The two calls the workload generators make on a handle (info, decode_points), answered from
    the oracle's own reading of an index directory: the same boxes and points as the product arm
    (both decode the same files, one rounded multiply per level), without loading the product."""

    def __init__(self, oracle, oidx):
        self.oidx = oidx
        self.pts, self.ids = oracle.decoded_points(oidx)

    def info(self):
        return {"N": int(self.pts.shape[0]), "D": int(self.oidx.D), "height": int(self.oidx.height)}

    def decode_points(self, positions):
        p = np.asarray(positions, dtype=np.int64)
        return self.pts[p], self.ids[p]


def cpu_brute_qps(oracle, pts, ids, qtype, queries, K=0, budget_s=15.0, first=16):
    """The FP64 brute-force scan (oracle.brute_query: every decoded point against every query, OpenMP
    over points on all host cores) timed over a bounded prefix of the workload: `first` queries, then
    doubled while the budget lasts. Returns (queries/s, cores, queries timed, their results)."""
    threads = os.cpu_count() or 1
    n, done, elapsed, res = min(first, len(queries)), 0, 0.0, None
    while done < len(queries):
        t0 = time.perf_counter()
        r = oracle.brute_query(pts, ids, qtype, queries[done:done + n], K=K, threads=threads)
        elapsed += time.perf_counter() - t0
        if res is None:
            res = (done, r)  # the first block's results (checked against the GPU's)
        done += n
        if elapsed * 3 > budget_s:
            break
        n = min(len(queries) - done, 2 * n)
    return done / elapsed, threads, done, res[1]


def knn_k(nq):
    """K of the batched-KNN workload: 20 for even queries, 100 for odd ones."""
    return np.where(np.arange(nq) % 2 == 0, 20, 100).astype(np.uint32)


def knn_legs(tb, h, P, K, steps, warmup, flush, n_plain=64):
    """Exact KNN over one index: the batched traversal with the learned ranking (timed steps), the
    same with the lower-bound ranking and with a one-pass finest level (three steps each, the median
    step reported), one query at
    a time with the lower-bound ranking and the scorer off (the plain traversal), and the learned
    batch end to end through the host-buffer entry point. Each batch is one synchronous C-ABI call,
    timed on the host with the device synchronised on both sides (L2 flushed before each step)."""
    import torch
    nq, D = P.shape
    dP = torch.from_numpy(P).cuda()

    def batch_leg(two_wave, learned, n_steps, n_warm, nvtx=None, median=False):
        h.set_two_wave(two_wave)
        h.scorer_enable(learned)
        for _ in range(max(1, n_warm)):  # the first batch sizes every workspace
            h.query_batch(tb.QueryType.POINT, dP, tb.Mode.EXACT, K=K)
        ts = []
        if nvtx:
            torch.cuda.nvtx.range_push(nvtx)  # profilers select these steps by the range
        runs, launches = [], 0
        for _ in range(n_steps):
            flush.zero_()
            torch.cuda.synchronize()
            l0 = tb.kernel_launches()
            t1 = time.perf_counter()
            h.query_batch(tb.QueryType.POINT, dP, tb.Mode.EXACT, K=K)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t1)
            launches += tb.kernel_launches() - l0
            runs.append(h.knn_batch_info()["runs"])
        if nvtx:
            torch.cuda.nvtx.range_pop()
        c = h.knn_counters()
        info = dict(h.knn_batch_info(), device_free_gb=torch.cuda.mem_get_info()[0] / 1e9,
                    library_device_gb=tb.lib().tblaeq_live_device_bytes() / 1e9, runs_per_step=runs,
                    step_ms=[round(t * 1e3, 3) for t in ts], gpu_launches=launches)
        if median:  # the comparison legs: the median step, so one slow step on a busy host does not decide
            return nq / statistics.median(ts), c["rows"] / nq, ts, info
        return nq * n_steps / sum(ts), c["rows"] / nq, ts, info

    learned_qps, learned_rows, step_s, learned_info = batch_leg(True, True, steps, warmup, nvtx="knn_timed")
    r = h.query_batch(tb.QueryType.POINT, dP, tb.Mode.EXACT, K=K)
    result = (r.offsets.numpy().copy(), r.ids.numpy().copy(), r.dist2.numpy().copy())
    lb_qps, lb_rows, _, lb_info = batch_leg(True, False, 3, 1, median=True)
    one_qps, one_rows, _, one_info = batch_leg(False, False, 3, 1, median=True)

    # The plain traversal: one query at a time, lower-bound ranking, scorer off.
    h.set_two_wave(True)
    h.scorer_enable(False)
    n_plain = min(n_plain, nq)
    for i in range(8):
        h.query_batch(tb.QueryType.POINT, dP[i:i + 1], tb.Mode.EXACT, K=K[i:i + 1])
    lat = []
    for i in range(n_plain):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        h.query_batch(tb.QueryType.POINT, dP[i:i + 1], tb.Mode.EXACT, K=K[i:i + 1])
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - t1)
    plain_qps = n_plain / sum(lat)

    # End to end: host points in, offsets + ids + squared distances out (learned ranking). One
    # untimed call first: a leg before may have split (and released the workspace), so the first
    # call can be the one that grows it again.
    h.set_two_wave(True)
    h.scorer_enable(True)
    h.query_batch_host(tb.QueryType.POINT, P, tb.Mode.EXACT, K=K, ids_cap=int(K.sum()))
    e2e_t, tot = [], 0
    for _ in range(max(1, steps)):
        t1 = time.perf_counter()
        offs, ids_h, d2 = h.query_batch_host(tb.QueryType.POINT, P, tb.Mode.EXACT, K=K, ids_cap=int(K.sum()))
        e2e_t.append(time.perf_counter() - t1)
        tot = len(ids_h)
    pl = sorted(x * 1e3 for x in lat)
    st = sorted(x * 1e3 for x in step_s)
    return {
        "value": learned_qps, "unit": "queries/s", "steps": len(step_s),
        "gpu_launches": learned_info["gpu_launches"],
        "ms_per_step": statistics.mean(step_s) * 1e3,
        "latency_ms": {"batch_p50": st[len(st) // 2], "batch_p99": st[min(len(st) - 1, int(len(st) * 0.99))],
                       "plain_query_p50": pl[len(pl) // 2], "plain_query_p99": pl[min(len(pl) - 1, int(len(pl) * 0.99))]},
        "e2e": {"value": nq * len(e2e_t) / sum(e2e_t), "unit": "queries/s",
                "h2d_bytes_per_step": nq * D * 8 + nq * 4, "d2h_bytes_per_step": (nq + 1) * 8 + tot * 16},
        "ranking": {"learned": {"qps": learned_qps, "rows_per_query": learned_rows, "traversal": learned_info},
                    "lower_bound": {"qps": lb_qps, "rows_per_query": lb_rows, "traversal": lb_info},
                    "one_pass": {"qps": one_qps, "rows_per_query": one_rows, "traversal": one_info}},
        "plain": {"value": plain_qps, "unit": "queries/s", "queries": n_plain,
                  "kind": "one query at a time, lower-bound ranking, scorer off",
                  "speedup_batched_learned_vs_plain": learned_qps / plain_qps},
    }, result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["batched", "small", "knn", "serving", "build"], default="batched")
    ap.add_argument("--build-n", type=int, default=50_000_000, help="build: points")
    ap.add_argument("--serve-requests", type=int, default=2000, help="serving: requests per offered load")
    ap.add_argument("--train-queries", type=int, default=2048, help="knn: separately seeded scorer training queries")
    ap.add_argument("--nq", type=int, default=4096)
    ap.add_argument("--plain-queries", type=int, default=512)
    ap.add_argument("--knn-queries", type=int, default=4096, help="batched: points of the KNN leg")
    ap.add_argument("--knn-steps", type=int, default=10, help="batched: timed steps of the KNN leg")
    ap.add_argument("--no-knn", action="store_true", help="batched: skip the KNN leg")
    ap.add_argument("--knn-probe", type=int, default=-1,
                    help="KNN: probe beam (clusters per query per level before wave 1; 0 = no probe; "
                         "-1 = the library's default)")
    ap.add_argument("--knn-completion", type=int, choices=[0, 1], default=1,
                    help="KNN: 1 = node-major completion after wave 1, 0 = the query-major wave 2")
    ap.add_argument("--knn-chunk", type=int, default=0, help="KNN: queries per traversal (0 = automatic)")
    ap.add_argument("--knn-refine", type=int, default=-1,
                    help="KNN: stride of the bound-refinement sample (0 = off; -1 = the library's default)")
    ap.add_argument("--knn-refine-stages", type=int, default=0,
                    help="KNN: refinement stages (1..4; 0 = the library's default)")
    ap.add_argument("--knn-wave1", type=float, default=0.0,
                    help="KNN: wave-1 scale (clusters = ceil(scale*K/leaf)+1, 2..32; 0 = the library's default)")
    ap.add_argument("--variants", default=None,
                    help="range configs: launch variant per level (0 direct, 1 staged, 2 node-major), comma "
                         "list; skips the autotuner (A/B timing, profiling one kind of kernel)")
    ap.add_argument("--no-float-points", action="store_true",
                    help="range configs: finest level tests every point in FP64 (no float copy first)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--policy", default="L0",
                    help="range configs: level policy, one for every interval or a comma list (L2/L3 read "
                         "an interval's rows from mapped host memory)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        tb, wl = None, _workloads()  # the reference arm never imports the product package
    else:
        tb = _package()
        wl = sys.modules.get("tblaeq_b200.workloads") or __import__("tblaeq_b200.workloads").workloads
    cfg_name = args.config
    if cfg_name == "build":
        return run_build(args, tb, rank, world, local)
    cfg = wl.CONFIGS[cfg_name]
    if cfg_name == "small":
        boxes_kw = dict(half_width=0.05)
    else:
        boxes_kw = dict(log_uniform=(0.001, 0.1))
    config = {"workload": f"{cfg_name} range: RandomKmeans N={cfg['N']} D={cfg['D']} ratios "
                          f"{','.join(map(str, cfg['ratios']))} seed {cfg['seed']} sigma/{cfg['sigma_divisor']}; "
                          f"{args.nq} boxes, half-widths "
                          + ("log-uniform [0.1%,10%]" if cfg_name != "small" else "5%") + " of extent",
              "index_points": cfg["N"], "dim": cfg["D"], "queries_per_step": args.nq, "mode": "exact",
              "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas{world}"}

    if cfg_name == "knn":
        return run_knn(args, tb, wl, rank, world, local)
    if cfg_name == "serving":
        return run_serving(args, tb, wl, rank, world, local)
    if args.impl == "reference":
        return run_reference(args, wl, cfg_name, config, rank, world)

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    tb.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    h = wl.generate_index(tb.QueryHandler, cfg_name)
    policy = [tb.LevelPolicy[p.strip().upper()] for p in args.policy.split(",")]
    if len(policy) == 1:
        policy = policy * h.info()["intervals"]
    h.prepare_for_query(policy)
    finest_streamed = policy[-1] in (tb.LevelPolicy.L2, tb.LevelPolicy.L3)
    if args.no_float_points:
        h.set_float_points(False)
    # The finest level decides points from their float copies (4·D bytes) where the library has them.
    float_points = not args.no_float_points and not finest_streamed and cfg["D"] in (4, 8, 16)
    config["finest_points"] = "float32 copy, FP64 near faces" if float_points else "FP64 rows"
    if args.policy != "L0":
        config["policy"] = [p.name for p in policy]
    Q = wl.range_boxes(h, args.nq, seed=42, **boxes_kw)
    dQ = torch.from_numpy(Q).cuda()
    D = cfg["D"]
    flags = 0 if args.no_graph else tb.USE_GRAPH

    # Warm-up: the first synchronous batch sizes every workspace, the autotuner picks a kernel
    # variant per level on this batch, the rest replay the graph.
    h.query_batch(tb.QueryType.RANGE, dQ, tb.Mode.EXACT)
    import tempfile
    cache = os.environ.get("TBLAEQ_TUNING_CACHE", os.path.join(tempfile.gettempdir(), "tblaeq_tuning.txt"))
    if args.variants:
        variants = [int(v) for v in args.variants.split(",")]
        grids, tuned_ms, tuned_from = [100] * len(variants), None, "--variants"
        h.set_launch_shapes(variants, grids)
    else:
        variants, grids, tuned_ms, tuned_from = h.autotune_cached(dQ, cache, tb.Mode.EXACT, reps=5)
    h.set_timing(True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        h.query_batch_async(tb.QueryType.RANGE, dQ, tb.Mode.EXACT, flags=flags)
        h.batch_wait()

    entries, items, results = h.level_counts()
    groups = h.group_counts()
    step_ms, final_ms, stage_rows = [], [], []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")  # profilers select the timed steps by this range
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            h.query_batch_async(tb.QueryType.RANGE, dQ, tb.Mode.EXACT, flags=flags)
            h.batch_wait()
            st = h.stage_times()
            step_ms.append(sum(st))
            final_ms.append(st[-2])
            stage_rows.append(st)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    if world > 1:
        dist.barrier()
    total_ms = max_over_ranks(sum(step_ms))
    value = job_throughput(args.nq * args.steps, world, total_ms / 1e3)
    # Kernels per step, counted from the nodes of the captured graph (one untimed capture when the
    # timed steps ran without one).
    graph = h.graph_launches()
    if not graph["kernels"]:
        h.query_batch_async(tb.QueryType.RANGE, dQ, tb.Mode.EXACT, flags=tb.USE_GRAPH)
        h.batch_wait()
        graph = h.graph_launches()

    # Roofline of the dominant level (largest event time): its algorithmic bytes per launch.
    H = len(entries)

    def level_bytes(m):
        """Bytes level m must move: per input entry its query slot, first child, prefix and
        coordinates (12 + 8·D); per tested child its P row and node record (8·D + 16), or at the
        finest level its point (float copy 4·D, FP64 row 8·D); per surviving entry the same entry
        fields written; per result its id and query slot (16). With point groups the finest level
        reads, per (query, cluster) entry, its groups' boxes and records (8·D + 16 each), and per
        kept (query, group) pair the points of the group."""
        if m < H - 1:
            if m < len(variants) and variants[m] == 2 and m > 0:
                # Node-major: every unit (a node and up to 32 of its entries) reads the node's
                # children once (float box 8·D, row 8·D, record 16), not once per entry.
                per_node = items[m] / max(1, entries[m])
                units = entries[m] / 32 + mesh_nodes[m - 1] / 2
                return (entries[m] * (12 + 8 * D) + units * per_node * (16 * D + 16)
                        + entries[m + 1] * (12 + 8 * D))
            return entries[m] * (12 + 8 * D) + items[m] * (8 * D + 16) + entries[m + 1] * (12 + 8 * D)
        if groups["groups"]:
            return (entries[m] * (12 + 8 * D) + groups["groups"] * (8 * D + 16) + groups["kept"] * 2 * (12 + 8 * D)
                    + groups["points"] * 4 * D + results * 16)
        return entries[m] * (12 + 8 * D) + items[m] * (4 if float_points else 8) * D + results * 16

    mesh_nodes = h.info()["meshSizes"][::-1]  # coarsest mesh first
    level_ms = [statistics.mean(r[1 + m] for r in stage_rows) for m in range(H)]
    dom = max(range(H), key=lambda m: level_ms[m])
    alg_bytes = level_bytes(dom)
    final_mean_s = level_ms[dom] / 1e3
    peak, peak_kind = _peaks()
    achieved = alg_bytes / final_mean_s / 1e9
    per_level = [{"level": m, "ms": level_ms[m], "algorithmic_bytes": level_bytes(m),
                  "GB/s": level_bytes(m) / (level_ms[m] / 1e3) / 1e9} for m in range(H)]
    dom_kind = (["direct", "staged", "node-major"][variants[dom]] if dom < len(variants) else "direct")
    dom_name = ("finest level: point groups + float points" if dom == H - 1 and groups["groups"]
                else "finest level" if dom == H - 1 else f"level {dom} (mesh {dom - 1} -> mesh {dom}), {dom_kind}")

    # Plain: one query at a time through the same engine (no batching, no graph).
    plain_lat = []
    n_plain = min(args.plain_queries, args.nq)
    for i in range(8):
        h.query_batch(tb.QueryType.RANGE, dQ[i:i + 1], tb.Mode.EXACT)
    torch.cuda.synchronize()
    for i in range(n_plain):
        t0 = time.perf_counter()
        h.query_batch(tb.QueryType.RANGE, dQ[i:i + 1], tb.Mode.EXACT)
        plain_lat.append(time.perf_counter() - t0)
    plain_qps = n_plain / sum(plain_lat)

    # End to end through the public host API with pinned host buffers.
    hostQ = torch.from_numpy(Q).pin_memory()
    cap = max(1024, int(results * 1.5) + 1024)
    offs_h = torch.empty(args.nq + 1, dtype=torch.int64).pin_memory()
    ids_h = torch.empty(cap, dtype=torch.int64).pin_memory()
    import ctypes
    lib = tb.lib()
    # Host boxes in, offsets and ids out, launches replayed from the handle's CUDA graph (the public
    # batch flag a serving caller would set).
    b = tb._Batch(int(tb.QueryType.RANGE), int(tb.Mode.EXACT), args.nq, hostQ.data_ptr(), 0, 0, flags, None)
    tot = ctypes.c_uint64()
    P64 = ctypes.POINTER(ctypes.c_uint64)
    def e2e_call():
        code = lib.tblaeq_query_batch_host(h._h, ctypes.byref(b), ctypes.cast(offs_h.data_ptr(), P64),
                                           ctypes.cast(ids_h.data_ptr(), P64), cap, None, ctypes.byref(tot))
        if code:
            raise tb.TblaeqError(code, lib.tblaeq_last_error().decode())
    # Untimed warm-up: the first few hundred host-path calls of a process run slower (measured on
    # B200: 1.4 against 0.87 ms per call), so the e2e leg warms up longer than the device leg, and
    # without the per-stage event timing the device leg needed.
    h.set_timing(False)
    for _ in range(max(args.warmup, 300)):
        e2e_call()
    e2e_t = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_call()
        e2e_t.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(sum(e2e_t))
    e2e_value = job_throughput(args.nq * args.steps, world, e2e_total)

    # The batched-plus-learned KNN leg on the same index: batched + learned exact queries against
    # the plain one-query-at-a-time traversal, at N = 10M, D = 8.
    knn, knn_result, Pk, Kk = None, None, None, None
    if cfg_name == "batched" and not args.no_knn:
        Pk = wl.knn_points(h, args.knn_queries, seed=1234, noise=0.02)
        Kk = knn_k(args.knn_queries)
        kcfg = {}
        knn_options(h, args, kcfg)
        T = wl.knn_points(h, 2048, seed=4321, noise=0.02)
        t0 = time.perf_counter()
        losses = h.scorer_train(T, K=knn_k(2048), max_samples=200000, epochs=8, lr=3e-3, seed=9)
        train_s = time.perf_counter() - t0
        with ClockSampler(local) as kclk:
            knn, knn_result = knn_legs(tb, h, Pk, Kk, args.knn_steps, args.warmup, flush)
        knn["value"] = knn["value"] * world
        knn["config"] = {"workload": f"knn on the same index: {args.knn_queries} points (data + N(0,(2% extent)^2)), "
                                     "K=20 and K=100 alternating", "queries_per_step": args.knn_queries, **kcfg}
        knn["scorer"] = {"train_queries": 2048, "train_s": train_s, "epoch_loss": losses, **h.scorer_stats()}
        knn["clocks"] = kclk.summary()

    cpu, port, agreement = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, REPO)
        import oracle
        pts, pids = h.decode_points(np.arange(h.info()["N"], dtype=np.uint64))
        qps, cores, sampled, bres = cpu_brute_qps(oracle, pts, pids, oracle.RANGE, Q)
        cpu = {"value": qps, "unit": "queries/s", "cores": cores, "kind": "port",
               "sample": f"first {sampled} of the {args.nq} boxes, FP64 brute-force scan of all {len(pts)} "
                         f"decoded points (lo <= x <= hi), OpenMP over points"}
        # The scan's results are the exact answers: the batched GPU results must equal them.
        n_chk = len(bres.offsets) - 1
        r = h.query_batch(tb.QueryType.RANGE, Q[:n_chk], tb.Mode.EXACT)
        go, gi = r.offsets.numpy(), r.ids.numpy()
        same = bool(np.array_equal(go, bres.offsets)) and all(
            np.array_equal(np.sort(gi[go[q]:go[q + 1]]), bres.query(q)) for q in range(n_chk))
        agreement = {"range": {"queries": n_chk, "identical_to_fp64_brute_force": same}}
        oidx = oracle_index_from_handler(oracle, h)
        sub = oracle.subtree(oidx)
        pqps, pcores, psampled = cpu_port_qps(oracle, oidx, sub, Q)
        port = {"value": pqps, "unit": "queries/s", "cores": pcores, "kind": "port",
                "sample": f"first {psampled} of the {args.nq} boxes, exact traversal port (subtree radii + "
                          f"final filter), OpenMP over queries"}
        if knn is not None:
            kq, kcores, ksampled, kres = cpu_brute_qps(oracle, pts, pids, oracle.KNN, Pk[:64][Kk[:64] == 20], K=20,
                                                       budget_s=8.0, first=8)
            knn["cpu_baseline"] = {"value": kq, "unit": "queries/s", "cores": kcores, "kind": "port",
                                   "sample": f"{ksampled} of the K=20 points, FP64 brute-force scan of all points"}
            ko, ki, kd = knn_result
            sel = np.nonzero(Kk[:64] == 20)[0][:len(kres.offsets) - 1]
            ok = all(np.array_equal(ki[ko[q]:ko[q + 1]], kres.query(j)) and
                     np.array_equal(kd[ko[q]:ko[q + 1]], kres.dist2[kres.offsets[j]:kres.offsets[j + 1]])
                     for j, q in enumerate(sel))
            agreement["knn"] = {"queries": len(sel), "identical_to_fp64_brute_force": bool(ok)}
        del pts, pids

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    lat_ms = sorted(step_ms)
    pl = sorted(x * 1e3 for x in plain_lat)
    out = {
        "metric": "exact-result range queries/s (batched, 1 B200 per rank)",
        "value": value,
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded RandomKmeans-style index and boxes)",
        "config": config,
        "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": args.nq * 2 * D * 8,
                "d2h_bytes_per_step": (args.nq + 1) * 8 + int(tot.value) * 8},
        # per step: the kernel nodes of the replayed graph (root frontier, box rounding, the level
        # kernels, transposes, headers, scans, result grouping)
        "gpu_launches": args.steps * graph["kernels"],
        "graph_nodes_per_step": graph,
        "latency_ms": {"batch_p50": lat_ms[len(lat_ms) // 2], "batch_p99": lat_ms[min(len(lat_ms) - 1,
                                                                                     int(len(lat_ms) * 0.99))],
                       "plain_query_p50": pl[len(pl) // 2], "plain_query_p99": pl[min(len(pl) - 1,
                                                                                       int(len(pl) * 0.99))]},
        "plain": {"value": plain_qps, "unit": "queries/s", "queries": n_plain,
                  "speedup_batched_vs_plain": value / world / plain_qps},
        "results_per_step": results,
        "autotune": {"variants": [["direct", "staged", "node-major"][v] for v in variants], "grid_percent": grids,
                     "level_ms": tuned_ms, "source": tuned_from, "cache": cache,
                     "searched": "variant {direct, staged, node-major} x persistent grid {100, 75, 50, 25}% of "
                                 "occupancy, per level, on the live batch"},
        "level_entries": entries,
        "level_children": items,
        # A finest interval read from mapped host memory is bound by the host link, not HBM.
        "roofline": {"bound": "host link" if finest_streamed else "hbm", "achieved": achieved,
                     "peak": None if finest_streamed else peak, "unit": "GB/s",
                     "frac": None if finest_streamed else achieved / peak,
                     "traffic": None if finest_streamed else profiled_traffic(cfg_name, args.nq, dom, H),
                     "kernel": dom_name,
                     "peak_kind": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": alg_bytes,
                     "launch_ms": final_mean_s * 1e3, "per_level": per_level, "point_groups": groups},
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "cpu_traversal_port": port,
        "agreement": agreement,
    }
    if knn is not None:
        out["knn"] = knn
        out["target"] = {
            "workload": "N=10M, D=8 (one index): 4096 range boxes and 4096 KNN points",
            "range_batched_vs_plain": value / world / plain_qps,
            "knn_batched_learned_vs_plain": knn["plain"]["speedup_batched_learned_vs_plain"],
            "dominant_level_hbm_frac": None if finest_streamed else achieved / peak,
            "needs": ">= 5x batched+learned vs plain, >= 0.60 of HBM in pruning/SpTSpM"}
    print(json.dumps(out))


def knn_workload(tb, wl, nq, seed):
    """KNN workload of the batched-KNN configuration: data points + N(0, (2% extent)^2) noise per
    dimension, alternating K=20 and K=100 (half of each)."""
    h = wl.generate_index(tb.QueryHandler, "knn")
    P = wl.knn_points(h, nq, seed=seed, noise=0.02)
    K = np.where(np.arange(nq) % 2 == 0, 20, 100).astype(np.uint32)
    return h, P, K


def knn_options(h, args, config):
    """Applies the KNN command-line options to a prepared handle and names them in `config`."""
    if args.knn_probe >= 0 or args.knn_completion != 1:
        beam = args.knn_probe if args.knn_probe >= 0 else 32
        h.set_knn_probe(beam, bool(args.knn_completion))
        config["knn_probe"] = {"beam": beam, "node_major_completion": bool(args.knn_completion)}
    if args.knn_chunk:
        h.set_knn_chunk(args.knn_chunk)
        config["knn_chunk"] = args.knn_chunk
    if args.knn_refine >= 0:
        h.set_knn_refine(args.knn_refine)
        config["knn_refine_stride"] = args.knn_refine
    if args.knn_refine_stages > 0:
        h.set_knn_refine_stages(args.knn_refine_stages)
        config["knn_refine_stages"] = args.knn_refine_stages
    if args.knn_wave1 > 0:
        h.set_knn_wave1(args.knn_wave1)
        config["knn_wave1_scale"] = args.knn_wave1


def run_knn(args, tb, wl, rank, world, local):
    """Batched exact KNN (N=50M, D=16, 4096 queries, K in {20, 100}) with the learned frontier
    ranking, beside the lower-bound ranking, the one-pass finest level and one query at a time.
    Each step is one synchronous batch through the C ABI, timed on the host around the call,
    synchronised on both sides. Replicas only for N > 1."""
    cfg = wl.CONFIGS["knn"]
    config = {"workload": f"knn: RandomKmeans N={cfg['N']} D={cfg['D']} ratios "
                          f"{','.join(map(str, cfg['ratios']))} seed {cfg['seed']} sigma/{cfg['sigma_divisor']}; "
                          f"{args.nq} points (data + N(0,(2% extent)^2)), K=20 and K=100 alternating",
              "index_points": cfg["N"], "dim": cfg["D"], "queries_per_step": args.nq, "mode": "exact",
              "l2": "inputs larger than L2 (6.4 GB of rows per step)", "parallelism": f"replicas{world}"}
    steps = args.steps if args.steps != 200 else 3
    metric = "exact-result KNN queries/s (batched + learned ranking, 1 B200 per rank)"
    if args.impl == "reference":
        if rank != 0:
            return
        sys.path.insert(0, REPO)
        import oracle
        view, _ = reference_index(oracle, "knn")
        P = wl.knn_points(view, args.nq, seed=1234, noise=0.02)
        K = knn_k(args.nq)
        per, t = 4, 0.0
        threads = os.cpu_count() or 1
        for s in range(steps):
            sl = slice((s * per) % args.nq, (s * per) % args.nq + per)
            t0 = time.perf_counter()
            for kv in (20, 100):
                m = K[sl] == kv
                if m.any():
                    oracle.brute_query(view.pts, view.ids, oracle.KNN, P[sl][m], K=kv, threads=threads)
            t += time.perf_counter() - t0
        v = per * steps / t
        print(json.dumps({"metric": metric, "value": v, "unit": "queries/s", "impl": "reference", "n_gpus": world,
                          "steps": steps, "warmup": 0, "ms_per_step": t / steps * 1e3, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": config,
                          "cpu_baseline": {"value": v, "unit": "queries/s", "cores": threads, "kind": "port",
                                           "sample": f"{per} points per step, FP64 brute force over all {cfg['N']} "
                                                     f"points (the reference's KNN is approximate; exact needs a scan)"},
                          "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    import torch
    torch.cuda.set_device(local)
    tb.set_device(local)
    h, P, K = knn_workload(tb, wl, args.nq, seed=1234)
    h.prepare_for_query(tb.LevelPolicy.L0)
    knn_options(h, args, config)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # Scorer: trained on traces of separately seeded queries (up to 200,000 samples).
    T = wl.knn_points(h, args.train_queries, seed=4321, noise=0.02)
    t0 = time.perf_counter()
    losses = h.scorer_train(T, K=knn_k(args.train_queries), max_samples=200000, epochs=8, lr=3e-3, seed=9)
    train_s = time.perf_counter() - t0
    stats = h.scorer_stats()
    with ClockSampler(local) as clk:
        leg, (ko, ki, kd) = knn_legs(tb, h, P, K, steps, args.warmup, flush, n_plain=min(args.plain_queries, 32))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, REPO)
        import oracle
        pts, ids = h.decode_points(np.arange(cfg["N"], dtype=np.uint64))
        threads = os.cpu_count() or 1
        t1 = time.perf_counter()
        for kv in (20, 100):
            oracle.brute_query(pts, ids, oracle.KNN, P[:4][K[:4] == kv], K=kv, threads=threads)
        cpu = {"value": 4 / (time.perf_counter() - t1), "unit": "queries/s", "cores": threads, "kind": "port",
               "sample": "the first 4 points, FP64 brute force over all points, OpenMP over points"}
    if rank != 0:
        return
    print(json.dumps({
        "metric": metric, "value": leg["value"] * world, "unit": "queries/s", "n_gpus": world, "steps": steps,
        "warmup": max(1, args.warmup), "ms_per_step": leg["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded RandomKmeans-style index and points)", "config": config,
        "e2e": leg["e2e"], "gpu_launches": leg["gpu_launches"], "latency_ms": leg["latency_ms"], "ranking": leg["ranking"],
        "plain": leg["plain"],
        "scorer": {"train_queries": args.train_queries, "samples": stats["samples"], "positives": stats["positives"],
                   "train_s": train_s, "epoch_loss": losses},
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }))


def serving_stream(h, wl, lam, n, seed, ext, pts_sample):
    """n requests of a Poisson stream at lam requests/s: half range boxes (half-widths log-uniform in
    [0.1%, 5%] of the extent), half KNN points (data + N(0, (1% extent)^2)) with K = floor(exp(U[0,
    ln 256])). Rows hold 2D values (KNN rows use the first D)."""
    rng = np.random.default_rng(seed)
    D = len(ext)
    at = np.cumsum(rng.exponential(1e6 / lam, n))
    qt = rng.integers(0, 2, n).astype(np.int32)
    c = pts_sample[rng.integers(0, len(pts_sample), n)]
    hw = np.exp(rng.uniform(np.log(0.001), np.log(0.05), (n, D))) * ext
    rows = np.concatenate([c - hw, c + hw], 1)
    knn = qt == 0
    rows[knn, :D] = (c + rng.normal(0, 1, (n, D)) * 0.01 * ext)[knn]
    rows[knn, D:] = 0
    K = np.where(knn, np.floor(np.exp(rng.uniform(0, np.log(256), n))), 0).astype(np.uint32)
    return qt, rows, K, at


def run_serving(args, tb, wl, rank, world, local):
    """Serving (N=100M, D=8): a Poisson stream of mixed range and KNN requests at swept offered
    loads, replayed at its arrival times into the continuous-batching server; p50/p99 latency from
    arrival to result and sustained completions/s per load, learned+batched vs one at a time."""
    cfg = wl.CONFIGS["serving"]
    config = {"workload": f"serving: RandomKmeans N={cfg['N']} D={cfg['D']} ratios "
                          f"{','.join(map(str, cfg['ratios']))} seed {cfg['seed']} sigma/{cfg['sigma_divisor']}; "
                          "Poisson arrivals, 50% range (half-widths log-uniform [0.1%,5%]), 50% KNN "
                          "(data + N(0,(1% extent)^2), K = floor(exp(U[0, ln 256])))",
              "index_points": cfg["N"], "dim": cfg["D"], "mode": "exact", "parallelism": f"replicas{world}"}
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference serves one request at a time "
                              "through its HTTP server, which is out of scope; its per-query CUDA path is timed "
                              "by tests/test_gpu_reference.py"}))
        return
    import torch
    torch.cuda.set_device(local)
    tb.set_device(local)
    h = wl.generate_index(tb.QueryHandler, "serving")
    h.prepare_for_query(tb.LevelPolicy.L0)
    lo_e, hi_e = wl.extent(h)
    ext = hi_e - lo_e
    D = cfg["D"]
    rng = np.random.default_rng(11)
    sample, _ = h.decode_points(rng.integers(0, cfg["N"], 200000).astype(np.uint64))
    T = sample[rng.integers(0, len(sample), 1024)] + rng.normal(0, 1, (1024, D)) * 0.01 * ext
    KT = np.floor(np.exp(rng.uniform(0, np.log(256), 1024))).astype(np.uint32)
    t0 = time.perf_counter()
    h.scorer_train(T, K=KT, max_samples=200000, epochs=8, lr=3e-3, seed=9)
    train_s = time.perf_counter() - t0
    h.scorer_enable(False)
    loads = [1e3, 1e4, 1e5, 1e6]

    def sweep(srv, loads, n_req, seed0):
        out = []
        qt, rows, K, at = serving_stream(h, wl, 1e3, 200, seed0, ext, sample)
        srv.replay(qt, rows, K, np.zeros(len(qt)))  # warm-up: sizes every lane's workspace
        srv.wait_idle(600000)
        srv.stats(reset=True)
        for j, lam in enumerate(loads):
            qt, rows, K, at = serving_stream(h, wl, lam, n_req, seed0 + 1 + j, ext, sample)
            tickets = srv.replay(qt, rows, K, at)
            srv.wait_idle(1800000)
            st = srv.stats(reset=True)
            for t in tickets:
                srv.poll(int(t), 0)
            out.append({"offered_qps": lam, "requests": n_req,
                        "sustained_qps": st["completed"] / st["span_s"] if st["span_s"] > 0 else None,
                        "p50_ms": st["p50_us"] / 1e3, "p99_ms": st["p99_us"] / 1e3, "mean_batch": st["mean_batch"],
                        "failed": st["failed"]})
        return out

    with ClockSampler(local) as clk:
        l0 = tb.kernel_launches()
        with tb.Server(h, max_batch=4096, learned=True) as srv:
            batched = sweep(srv, loads, args.serve_requests, 100)
        launches = tb.kernel_launches() - l0
    with tb.Server(h, max_batch=1, lanes=1, learned=False) as srv:
        plain = sweep(srv, [1e3, 1e4, 1e6], min(args.serve_requests, 400), 200)
    if rank != 0:
        return
    best = max(r["sustained_qps"] or 0 for r in batched)
    best_plain = max(r["sustained_qps"] or 0 for r in plain)
    print(json.dumps({
        "metric": "exact-result queries/s served (continuous batching, learned ranking, 1 B200 per rank)",
        "value": best * world, "unit": "queries/s", "n_gpus": world, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded RandomKmeans-style index, Poisson stream)",
        "config": config,
        "e2e": {"value": best * world, "unit": "queries/s", "note": "requests enter and leave on the host"},
        "gpu_launches": launches, "loads": batched, "plain_one_at_a_time": plain,
        "speedup_vs_plain_at_saturation": best / best_plain if best_plain else None, "scorer_train_s": train_s,
        "clocks": clk.summary()}))


def build_points(n, D=16, seed=2024):
    """The build configuration's points: 80% in 10,000 Gaussian clusters (sigma 0.01, centres
    uniform in [0,1]^D), 20% uniform in [0,1]^D, FP32, in random order."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, 1, (10000, D)).astype(np.float32)
    m = int(n * 0.8)
    X = np.empty((n, D), np.float32)
    step = 1 << 22
    for i in range(0, m, step):
        j = min(m, i + step)
        X[i:j] = centres[rng.integers(0, len(centres), j - i)] + rng.normal(0, 0.01, (j - i, D)).astype(np.float32)
    X[m:] = rng.uniform(0, 1, (n - m, D)).astype(np.float32)
    return X[rng.permutation(n)]


def run_build(args, tb, rank, world, local):
    """Index build (k-means hierarchy): N points, D=16 FP32, height 4, ratios 100,50,20, 20 Lloyd
    iterations per level, assignment on the tensor cores (tcgen05, 3xTF32). The objective is
    compared with the FP64 CUDA-core build from the same start on the first 2,000,000 points (an
    FP64 build of all points would take hours). Replicas only for N > 1."""
    D = 16
    config = {"workload": f"build: k-means hierarchy over {args.build_n} points (80% in 10,000 Gaussian clusters "
                          "sigma 0.01, 20% uniform, [0,1]^16, FP32), height 4, ratios 100,50,20, 20 Lloyd "
                          "iterations per level", "points": args.build_n, "dim": D,
              "parallelism": f"replicas{world}"}
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference builds with cuVS k-means, which is "
                              "not installed here; its CPU fallback is O(N k D) per iteration (days at this size)"}))
        return
    import torch
    torch.cuda.set_device(local)
    tb.set_device(local)
    X = build_points(args.build_n, D)
    with ClockSampler(local) as clk:
        l0 = tb.kernel_launches()
        t0 = time.perf_counter()
        h, rep = tb.QueryHandler.build(X, height=4, ratios=(100, 50, 20), iters=20, seed=1)
        total = time.perf_counter() - t0
        launches = tb.kernel_launches() - l0
    sub = min(args.build_n, 2_000_000)
    _, rt = tb.QueryHandler.build(X[:sub], height=4, ratios=(100, 50, 20), iters=20, seed=1)
    _, r64 = tb.QueryHandler.build(X[:sub], height=4, ratios=(100, 50, 20), iters=20, seed=1,
                                   precision=tb.KmeansPrecision.FP64)
    if rank != 0:
        return
    peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(REPO, "MEASURED_PEAKS.json")) else {}
    lvl0 = rep[0]
    # Tensor work of level 0: 3 TF32 products of a (n x 16) by (16 x k) GEMM per iteration.
    flops = 3 * 2.0 * lvl0["n"] * lvl0["k"] * 16 * lvl0["iters"]
    achieved = flops / lvl0["assign_seconds"] / 1e12
    tf32_peak = peaks.get("bf16_tflops", 1590.0) / 2
    # The algorithmic distance FLOPs (2 N k D per Lloyd iteration, one product per distance), against
    # the measured dense BF16 GEMM rate of a seconds-long loop (the assignment runs for seconds).
    alg = 2.0 * lvl0["n"] * lvl0["k"] * D * lvl0["iters"] / lvl0["assign_seconds"] / 1e12
    sustained = peaks.get("bf16_tflops_sustained", 1400.0)
    print(json.dumps({
        "metric": "index build: points indexed per second (k-means hierarchy, 1 B200 per rank)",
        "value": args.build_n / total * world, "unit": "points/s", "n_gpus": world, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "tf32x3 (fp32 accumulate)", "data": "synthetic",
        "config": config, "seconds": total, "gpu_launches": launches,
        "levels": rep,
        "objective_vs_fp64": {"points": sub, "tensor": [r["objective"] for r in rt],
                              "fp64": [r["objective"] for r in r64],
                              "rel_diff": [abs(a["objective"] - b["objective"]) / b["objective"]
                                           for a, b in zip(rt, r64)]},
        "roofline": {"bound": "tensor", "kernel": "assignTcKernel (level 0)", "achieved": achieved,
                     "peak": tf32_peak, "unit": "TFLOP/s", "frac": achieved / tf32_peak,
                     "peak_kind": "half the measured bf16 dense GEMM (TF32 rate)",
                     "note": "3 TF32 products per distance; the per-point argmin epilogue on CUDA cores bounds it",
                     "algorithmic": {"achieved": alg, "unit": "TFLOP/s", "flops_per_iteration": 2.0 * lvl0["n"] * lvl0["k"] * D,
                                     "peak": sustained, "frac": alg / sustained,
                                     "peak_kind": ("measured" if "bf16_tflops_sustained" in peaks else "fallback")
                                                  + " bf16_tflops_sustained"}},
        "assemble_seconds": [r["assemble_seconds"] for r in rep],
        "clocks": clk.summary()}))


def write_query_file(path, rows, D):
    """The reference's query-file format (src/Data_Structures/File.cu:159-205): a header "n D", then
    one row per query (2D values lo|hi for range, D values for a point), %.17g so values round-trip."""
    with open(path, "w") as f:
        f.write(f"{rows.shape[0]} {D}\n")
        for r in np.asarray(rows, dtype=np.float64):
            f.write(" ".join("%.17g" % v for v in r) + "\n")


def reference_cuda(idx_dir, Q, D, kind, K=0, timeout=1800):
    """The reference's own CUDA build (oracle/_ref/ref_harness: the reference's
    QueryHandler::performSingleRangeQuery / performSingleKNNQuery with saveFineMesh=true under policy
    L0) on this GPU, one query at a time, timed by its per-query timer; like its CLI
    (QueryEngine.cu:216-227) the mean drops the fastest and the slowest query. It returns the
    reference's candidate sets: every point of every surviving cluster, without an exact final
    filter or top-K."""
    harness = os.path.join(REPO, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return {"unavailable": "the reference build (oracle/_ref) is not present"}
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        # The reference labels a query file by the text after the last '_' of its path
        # (src/utils/Utils.cu:18-35): keep it free of '-'.
        qf = os.path.join(d, "q_" + kind + ".txt")
        write_query_file(qf, Q, D)
        out = os.path.join(d, "ref.bin")
        subprocess.run([harness, idx_dir, qf, "1" if kind == "knn" else "0", str(K), "L0", out], check=True,
                       timeout=timeout, stdout=subprocess.DEVNULL)
        us, cands = read_harness_times(open(out, "rb").read())
    t = sorted(us)
    mean = reference_mean_us(us)
    return {"value": 1e6 / mean, "unit": "queries/s", "queries": len(us), "mean_us": mean,
            "p50_us": t[len(t) // 2], "candidates": cands,
            "kind": f"reference CUDA build on this GPU, one {kind} query at a time, policy L0"
                    + (f", K={K}" if kind == "knn" else ""),
            "results": "the reference's candidate sets (no exact final filter)"}


def reference_index(oracle, wl, cfg_name):
    """The configuration's index as the reference's own generator writes it (oracle/_ref/T-BLAEQ
    --gen-index, default value range [1, 100]) in a temporary directory, read back by the oracle's
    reader: (workload view, directory). Neither step loads the product library."""
    import tempfile
    cfg = wl.CONFIGS[cfg_name]
    binary = os.path.join(REPO, "oracle", "_ref", "T-BLAEQ")
    if not os.path.exists(binary):
        raise FileNotFoundError("the reference build (oracle/_ref/T-BLAEQ) is not present")
    d = tempfile.mkdtemp(prefix="tblaeq_ref_idx_")
    subprocess.run([binary, "--gen-index", "-i", d, "--gen-N", str(cfg["N"]), "--gen-D", str(cfg["D"]),
                    "--height", str(len(cfg["ratios"]) + 1), "--ratios", ",".join(map(str, cfg["ratios"])),
                    "--gen-seed", str(cfg["seed"]), "--gen-sigma-divisor", str(cfg["sigma_divisor"])],
                   check=True, stdout=subprocess.DEVNULL, timeout=1800)
    return OracleWorkloadView(oracle, oracle.load_index(d)), d


def read_harness_times(raw: bytes):
    """Per-query microseconds and the total candidate count from the reference harness's dump:
    u64 query count, u64 interval count, then per query: interval u64 level sizes, f64 microseconds,
    u64 candidate count and that many u64 ids."""
    nq, intervals = (int(x) for x in np.frombuffer(raw, np.uint64, 2, 0))
    off, us, cands = 16, [], 0
    for _ in range(nq):
        off += 8 * intervals
        us.append(float(np.frombuffer(raw, np.float64, 1, off)[0]))
        off += 8
        c = int(np.frombuffer(raw, np.uint64, 1, off)[0])
        off += 8 + 8 * c
        cands += c
    if off != len(raw):
        raise ValueError("reference harness output has trailing or missing bytes")
    return us, cands


def reference_mean_us(us):
    """The reference CLI's per-query mean: the fastest and the slowest query dropped when there are
    more than two (src/core/QueryEngine.cu:216-227)."""
    t = sorted(us)
    kept = t[1:-1] if len(t) > 2 else t
    return sum(kept) / len(kept)


def run_reference(args, wl, cfg_name, config, rank, world):
    """Reference arm: the CPU restatement of the reference traversal (exact semantics) timed on the
    host cores over whole steps of the workload. The reference has no CPU implementation of its
    query path (every strategy launches CUDA kernels), so the oracle port stands in for it. The
    index comes from the reference's own generator and the oracle's reader, so this process never
    loads the product library. Beside it: the reference's own CUDA build, one query at a time on the
    same GPU (range, and KNN with K=20 and K=100), and the FP64 brute-force scan."""
    if rank != 0:
        return
    import shutil
    sys.path.insert(0, REPO)
    import oracle
    metric = "exact-result range queries/s (batched, 1 B200 per rank)"
    try:
        view, idx_dir = reference_index(oracle, wl, cfg_name)
    except Exception as e:
        print(json.dumps({"impl": "reference", "metric": metric, "unavailable": f"{type(e).__name__}: {e}"[:200]}))
        return
    try:
        oidx = view.oidx
        D = oidx.D
        boxes_kw = dict(half_width=0.05) if cfg_name == "small" else dict(log_uniform=(0.001, 0.1))
        Q = wl.range_boxes(view, args.nq, seed=42, **boxes_kw)
        sub = oracle.subtree(oidx)
        threads = os.cpu_count() or 1
        # Each step is the whole workload (all nq boxes), like the product arm's step.
        oracle.exact_query(oidx, oracle.RANGE, Q, sub=sub, threads=threads)  # untimed: first touch
        steps, t = 0, 0.0
        for s in range(max(1, args.steps)):
            t0 = time.perf_counter()
            oracle.exact_query(oidx, oracle.RANGE, Q, sub=sub, threads=threads)
            t += time.perf_counter() - t0
            steps += 1
            if t > 60.0:  # bounded: a slow host ends the arm after about a minute of timed work
                break
        v = args.nq * steps / t
        out = {"metric": metric, "value": v, "unit": "queries/s",
               "impl": "reference", "n_gpus": world, "steps": steps, "warmup": 1, "ms_per_step": t / steps * 1e3,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic (seeded RandomKmeans-style index written by the reference's --gen-index; boxes)",
               "config": config,
               "cpu_baseline": {"value": v, "unit": "queries/s", "cores": threads, "kind": "port",
                                "sample": f"all {args.nq} boxes per step ({steps} steps), exact traversal port, "
                                          f"OpenMP over queries"},
               "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        bq, bcores, bn, _ = cpu_brute_qps(oracle, view.pts, view.ids, oracle.RANGE, Q)
        out["cpu_brute_force"] = {"value": bq, "unit": "queries/s", "cores": bcores,
                                  "sample": f"first {bn} boxes, FP64 brute-force scan of all decoded points"}
        # The reference's own implementation runs on the GPU only.
        try:
            out["reference_cuda_b200"] = reference_cuda(idx_dir, Q[:min(args.nq, 256)], D, "range")
        except Exception as e:  # reported, never fatal to the CPU arm
            out["reference_cuda_b200"] = {"unavailable": f"{type(e).__name__}: {e}"[:200]}
        if cfg_name == "batched" and not args.no_knn:
            P = wl.knn_points(view, args.knn_queries, seed=1234, noise=0.02)
            K = knn_k(args.knn_queries)
            knn = {}
            for kv in (20, 100):
                try:
                    knn[f"K{kv}"] = reference_cuda(idx_dir, P[:256][K[:256] == kv], D, "knn", K=kv)
                except Exception as e:
                    knn[f"K{kv}"] = {"unavailable": f"{type(e).__name__}: {e}"[:200]}
            ok = [r["value"] for r in knn.values() if "value" in r]
            if len(ok) == 2:  # the mix of the workload: half K=20, half K=100
                knn["mixed"] = {"value": 2.0 / (1.0 / ok[0] + 1.0 / ok[1]), "unit": "queries/s"}
            out["reference_cuda_b200_knn"] = knn
        print(json.dumps(out))
    finally:
        shutil.rmtree(idx_dir, ignore_errors=True)


if __name__ == "__main__":
    main()
