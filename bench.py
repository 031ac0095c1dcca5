#!/usr/bin/env python
"""Graph500 BFS benchmark of the B200 engine.

Metric: harmonic-mean GTEPS of single-source direction-optimizing BFS on the
Graph500 Kronecker graph (SCALE 28, edgefactor 16, seeds 2/3), the quantity
main.cc prints as harmonic_mean_TEPS (mpi/main.cc:684-701, logfile.h:86-101):
TEPS_i = edge_visit_count_i / bfs_time_i, harmonic mean over the roots.
The graph is generated on the device (synthetic input of the benchmark's own
generator); roots come from find_roots with the re-pick rule of
find_roots_in_large_graph (main.cc:334-359); every root's parent array is
validated on the device before timing and its traversed-edge count is the
TEPS numerator.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one search from one root (the roots cycle).  N > 1 runs N
independent replicas (one graph per GPU; the search does not shard), launched
with torch.distributed.run; times are the max over ranks.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "graph500-bfs_b200"))


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=64)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--scale", type=int, default=28)
    p.add_argument("--edgefactor", type=int, default=16)
    p.add_argument("--roots", type=int, default=64)
    p.add_argument("--root-seed", type=int, default=0)
    p.add_argument("--alpha", type=float, default=10.0)
    p.add_argument("--beta", type=float, default=14.0)
    # The SCALE 28 workload runs as the reference's -A -C with degree-ordered
    # group reordering; each part can be switched off.
    p.add_argument("--no-corebfs", dest="corebfs", action="store_false",
                   help="without CoreBFS forest pruning (-C)")
    p.add_argument("--no-group-reorder", dest="group_reorder", action="store_false",
                   help="one global degree order instead of groups of 2^16 ids")
    p.add_argument("--no-auto-tune", dest="auto_tune", action="store_false",
                   help="without the -A alpha/beta tuner")
    p.add_argument("--no-tune-engine", dest="tune_engine", action="store_false",
                   help="keep the default kernel forms and batch alpha instead of timing them")
    p.add_argument("--no-tune-switch", dest="tune_switch", action="store_false",
                   help="keep alpha/beta as given (or as -A tuned them) instead of refining "
                        "them by timing in the engine tuner")
    p.add_argument("--batch-roots", type=int, default=64)
    p.add_argument("--batch-steps", type=int, default=20)
    p.add_argument("--batch-alpha", type=float, default=0.0,
                   help="alpha of the batched search (<= 0: the engine's batch default)")
    p.add_argument("--engine-option", action="append", default=[], metavar="NAME=VALUE",
                   help="set an engine option (b200bfs_set_option) before timing; repeatable")
    p.add_argument("--batch-sweep", action="store_true",
                   help="also time batches of 1, 8, 32 and 64 roots")
    p.add_argument("--batch-host-loop", action="store_true",
                   help="batched search with the host-driven level loop (for profilers that "
                        "cannot see kernels inside conditional CUDA graphs)")
    p.add_argument("--serve-rates", default="1000,10000,100000",
                   help="offered query rates (per s) of the serving leg")
    p.add_argument("--serve-seconds", type=float, default=1.5)
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--cpu-sample-sec", type=float, default=20.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--ref-scale", type=int, default=22,
                   help="SCALE of the reference arm (--impl reference): the reference's own "
                        "CPU program cannot build the SCALE 28 graph on this host")
    p.add_argument("--ref-timeout", type=float, default=1800.0)
    return p.parse_args()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        d = json.load(open(path))
        return d.get(kernel)
    except (OSError, ValueError):
        return None


def dist_setup(timeout_s=300):
    """One process per GPU (torch.distributed.run sets RANK/WORLD_SIZE/...):
    NCCL between the ranks' GPUs, gloo where CUDA is absent (host-side tests
    of the replica plumbing). Only the timing bookkeeping crosses ranks: the
    replicas share nothing else."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local, dist


def _reduce(dist, value, op):
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def barrier_max(dist, value):
    """Barrier, then the max of value over ranks."""
    if dist is None:
        return value
    return _reduce(dist, value, dist.ReduceOp.MAX)


def barrier_sum(dist, value):
    if dist is None:
        return value
    return _reduce(dist, value, dist.ReduceOp.SUM)


def build_flags(args):
    import b200bfs

    return (b200bfs.BUILD_COREBFS if args.corebfs else 0) | (
        b200bfs.BUILD_GROUP_REORDER if args.group_reorder else 0)


def pick_roots(eng, args):
    """find_roots + the re-pick rule of find_roots_in_large_graph
    (main.cc:334-359): roots are drawn again with the next seed while any of
    them reaches no more than 3 levels.  The depths (AUTO_LEVEL) come from
    one batched search per 64 roots (b200bfs_batch_root_levels, the value
    b200bfs_run reports for each root alone).  Each root's result is then
    validated on the device (validation level 2) and its traversed-edge count
    kept.  Returns the roots, their counts and the time of the first
    single-root search after prepare (pred and bitmaps cold)."""
    import torch

    r = args.root_seed
    while True:
        roots = eng.find_roots(args.roots, r, 0)
        depth = np.concatenate([(eng.run_batch(roots[i:i + 64], args.edgefactor, 0.0, args.beta),
                                 eng.batch_root_levels())[1] for i in range(0, len(roots), 64)])
        if args.scale <= 6 or (depth > 3).all():
            break
        log(f"root seed {r}: a root reaches <= 3 levels, picking roots again")
        r += 1
    stream = torch.cuda.ExternalStream(eng.stream())
    nedge, cold_ms = [], None
    for root in roots:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.run(int(root), args.edgefactor, args.alpha, args.beta)
        b.record(stream)
        b.synchronize()
        if cold_ms is None:
            cold_ms = a.elapsed_time(b)
        err, cnt = eng.validate(int(root))
        if err != 0:
            raise RuntimeError(f"validation failed for root {root}: {err} errors")
        nedge.append(cnt)
    return roots, np.array(nedge, dtype=np.float64), cold_ms


def td_random_access(eng, info, stats, td_ms, stream):
    """The top-down kernels against the random-access ceiling: probes per
    second (b200bfs_random_access_rate, loads and ORs into a buffer of the
    visited bitmap's size, rounded up to a power of two) and the probe-only
    time the searches' top-down entries would take at that rate."""
    import torch
    import b200bfs
    words = max(1, (info.num_rows + 31) // 32)
    log2w = max(10, (words - 1).bit_length())
    buf = torch.zeros(1 << log2w, dtype=torch.int32, device="cuda")
    loads = b200bfs.random_access_rate(buf.data_ptr(), log2w, 0, stream.cuda_stream)
    ors = b200bfs.random_access_rate(buf.data_ptr(), log2w, 1, stream.cuda_stream)
    del buf
    entries = sum(s.edges_scanned_td for s in stats)
    ceiling_ms = 1e3 * entries / loads
    return {"buffer_bytes": 4 << log2w, "loads_per_s": loads, "ors_per_s": ors,
            "entries_per_search": entries / len(stats),
            "entries_per_s": entries / (td_ms / 1e3) if td_ms > 0 else 0.0,
            "probe_ceiling_ms_per_search": ceiling_ms / len(stats),
            "frac": ceiling_ms / td_ms if td_ms > 0 else None}


def harmonic_teps(nedge, times):
    return len(times) / float(np.sum(np.asarray(times) / np.asarray(nedge)))


def cpu_search_sample(row_ptr, col, mdeg, inv, pred_size, rows, nedge, args, budget_sec):
    """Times the oracle's CPU restatement of the reference search on the
    benchmark graph for a bounded sample of roots."""
    import ctypes

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    L = O.lib()
    L.orc_bfs_csr32.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(O.BfsStats)]
    pred = np.empty(pred_size, dtype=np.int64)
    at = np.full(9, -1, dtype=np.int64)
    st = O.BfsStats()
    times, used = [], []
    t_start = time.perf_counter()
    for i, r in enumerate(rows):
        t0 = time.perf_counter()
        L.orc_bfs_csr32(row_ptr.shape[0] - 1, O._ptr(row_ptr), O._ptr(col), O._ptr(mdeg),
                        O._ptr(inv), pred_size, int(r), args.edgefactor, args.alpha, args.beta,
                        O._ptr(pred), O._ptr(at), ctypes.byref(st))
        times.append(time.perf_counter() - t0)
        used.append(nedge[i])
        if time.perf_counter() - t_start > budget_sec:
            break
    return times, used, O.num_threads()


def host_csr(eng):
    row_ptr, col, inv, mdeg = eng.get_csr()
    return row_ptr, col, inv, mdeg


def rows_of(inv, roots, nverts):
    """CSR rows of the given original vertex ids."""
    rank = np.full(nverts, -1, dtype=np.int64)
    rank[inv] = np.arange(inv.size, dtype=np.int64)
    return rank[np.asarray(roots, dtype=np.int64)]


def cpu_baseline_leg(args, device, roots, nedge):
    """The reference's plain CPU search (no -A, no -C: the default
    `mpiexec -n 1 runnable` run), restated by the oracle, timed on all host
    cores over a bounded sample of the same roots on the same generated graph
    (built on the device without pruning and copied to host memory)."""
    import b200bfs

    eng = b200bfs.Engine(device)
    eng.generate_graph(args.scale, args.edgefactor)
    info = eng.info()
    row_ptr, col, inv, mdeg = host_csr(eng)
    eng.close()
    rows = rows_of(inv, roots, 1 << info.scale)
    plain = argparse.Namespace(**vars(args))
    plain.alpha, plain.beta = 10.0, 14.0
    ct, cu, cores = cpu_search_sample(row_ptr, col, mdeg, inv, info.pred_size, rows, nedge,
                                      plain, args.cpu_sample_sec)
    return {"value": harmonic_teps(cu, ct) / 1e9, "unit": "GTEPS", "cores": cores, "kind": "port",
            "sample": f"{len(ct)} searches at SCALE {args.scale} (about {sum(ct):.0f} s) with the "
                      "oracle's OpenMP restatement of BfsBase::run_bfs_core (plain, alpha 10, "
                      "beta 14) on the same graph and roots"}


def percentile(x, q):
    return float(np.percentile(np.asarray(x, dtype=np.float64), q)) if len(x) else None


def batched_leg(eng, roots, nedge, args, stream, dist, single_times, single_pred_ms):
    """64-root batched search (b200bfs_run_batch) on the same graph: BFS/s of
    whole batches against the BFS/s of 64 sequential single-root runs, with
    batch latency percentiles.  Two baselines from the single-source searches
    timed above: as run (b200bfs_run writes each root's complete pred, the
    reference's output), and like for like with the batch, whose output is
    each root's levels: the same searches without their pred assembly pass
    (its CUDA-event time subtracted; the level kernels' row-order entries
    then hold each row's level and parent).  One root of the last batch is
    validated on the device."""
    import torch

    k = min(args.batch_roots, len(roots), 64)
    if args.batch_host_loop:
        eng.set_option("batch_graph", 0)
    for w in range(max(args.warmup, 3)):
        eng.run_batch(np.roll(roots, w)[:k], args.edgefactor, args.batch_alpha, args.beta)
    times, stats = [], None
    torch.cuda.synchronize()
    for b in range(args.batch_steps):
        sub = np.roll(roots, 7 * b)[:k]
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stats = eng.run_batch(sub, args.edgefactor, args.batch_alpha, args.beta)
        e.record(stream)
        e.synchronize()
        times.append(a.elapsed_time(e) / 1e3)
    idx = {int(r): i for i, r in enumerate(roots)}
    i_last = k // 2
    eng.batch_select(i_last)
    r_last = int(sub[i_last])
    err, cnt = eng.validate(r_last)
    if err != 0 or cnt != nedge[idx[r_last]]:
        raise RuntimeError(f"batched result for root {r_last} failed validation")
    sweep = []
    if args.batch_sweep:
        for kk in (1, 8, 32, 64):
            kk = min(kk, len(roots))
            ts = []
            for b in range(6):
                sub = np.roll(roots, 5 * b)[:kk]
                a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                eng.run_batch(sub, args.edgefactor, args.batch_alpha, args.beta)
                e.record(stream)
                e.synchronize()
                if b:  # the first is a warm-up
                    ts.append(a.elapsed_time(e) / 1e3)
            tk = barrier_max(dist, float(np.median(ts)))
            sweep.append({"roots_per_batch": kk, "batch_ms": 1e3 * tk,
                          "bfs_per_s": (dist.get_world_size() if dist else 1) * kk / tk})
    t_batch = barrier_max(dist, float(np.median(times)))
    t_single = barrier_max(dist, float(np.mean(single_times)))
    t_single_lo = barrier_max(dist, float(np.mean(np.asarray(single_times)
                                                  - np.asarray(single_pred_ms) / 1e3)))
    world = dist.get_world_size() if dist is not None else 1
    bfs_s = world * k / t_batch
    seq_bfs_s = world / t_single
    seq_lo_bfs_s = world / t_single_lo
    sub_nedge = [nedge[idx[int(r)]] for r in np.roll(roots, 0)[:k]]
    return {
        "roots_per_batch": k, "batches": args.batch_steps,
        "bfs_per_s": bfs_s, "sequential_single_root_bfs_per_s": seq_bfs_s,
        "speedup_vs_sequential": bfs_s / seq_bfs_s,
        "sequential_levels_only_bfs_per_s": seq_lo_bfs_s,
        "speedup_vs_sequential_levels_only": bfs_s / seq_lo_bfs_s,
        "baseline_definition": (
            "speedup_vs_sequential: against 64 sequential b200bfs_run searches, each writing its "
            "root's complete pred (2^SCALE int64 entries), as BfsBase::run_bfs does; "
            "speedup_vs_sequential_levels_only: against the same searches without the pred "
            "assembly pass, producing each root's levels like the batch"),
        "aggregate_gteps": world * float(np.sum(sub_nedge)) / t_batch / 1e9,
        "batch_ms_p50": 1e3 * percentile(times, 50), "batch_ms_p99": 1e3 * percentile(times, 99),
        "single_root_ms_p50": 1e3 * percentile(single_times, 50),
        "single_root_ms_p99": 1e3 * percentile(single_times, 99),
        "levels": stats.levels, "td_levels": stats.num_td_levels,
        "bu_levels": stats.num_bu_levels,
        "edges_scanned_per_input_edge": (stats.edges_scanned_td + stats.edges_scanned_bu)
        / max(1.0, float(eng.info().num_input_edges)),
        "algorithmic_gbs": stats.algorithmic_bytes / (stats.ms / 1e3) / 1e9,
        "level_loop": "CUDA graph (WHILE conditional node), one host sync per batch",
        "sweep": sweep or None,
    }


# The serving workload: Kronecker graphs of the benchmark's generator resident
# together, (SCALE, edgefactor).
SERVE_GRAPHS = [(16, 16), (18, 16), (20, 16), (22, 16), (24, 16), (22, 8), (22, 32)]


def serving_leg(args, device):
    """BFS serving with continuous batching (b200bfs_server_*): the graphs of
    SERVE_GRAPHS resident on the device under a 150 GB budget, (graph, root)
    queries arriving as a Poisson process (graph uniform, root uniform over a
    pool of 1024 vertices with edges per graph), for each offered rate.
    Latency is submit -> result on the device, measured by the server."""
    import b200bfs

    srv = b200bfs.Server(device, keep_results=False, slots_per_graph=2,
                         hbm_budget_bytes=150 * 10**9)
    out = {"graphs": [f"SCALE {s} ef {ef}" for s, ef in SERVE_GRAPHS], "rates": []}
    try:
        t0 = time.time()
        gids = [srv.add_graph(s, ef) for s, ef in SERVE_GRAPHS]
        pools = [srv.find_roots(g, 1024) for g in gids]
        out["build_s"] = time.time() - t0
        for g, pool in zip(gids, pools):  # one batch per graph and slot builds the graphs
            ids = [srv.submit(g, int(r)) for r in pool[:128]]
            for rid in ids:
                srv.wait(rid)
                srv.release(rid)
        rng = np.random.default_rng(12345)
        for lam in [float(x) for x in args.serve_rates.split(",") if x]:
            n = max(1, int(lam * args.serve_seconds))
            t_arr = np.cumsum(rng.exponential(1.0 / lam, n))
            gsel = rng.integers(0, len(gids), n)
            rsel = rng.integers(0, 1024, n)
            srv.reset_stats()
            start = time.perf_counter()
            for i in range(n):
                while time.perf_counter() - start < t_arr[i]:
                    pass
                srv.submit(gids[gsel[i]], int(pools[gsel[i]][rsel[i]]))
            t_sub = time.perf_counter() - start
            deadline = time.perf_counter() + 120
            while srv.stats().completed + srv.stats().failed < n and time.perf_counter() < deadline:
                time.sleep(0.005)
            st = srv.stats()
            out["rates"].append({
                "offered_per_s": lam, "submitted_per_s": n / t_sub, "requests": n,
                "completed": st.completed, "failed": st.failed, "bfs_per_s": st.bfs_per_s,
                "p50_ms": st.p50_ms, "p99_ms": st.p99_ms, "max_ms": st.max_ms,
                "mean_batch": st.mean_batch_size, "batches": st.batches})
            log(f"serving at {lam:.0f}/s: {st.bfs_per_s:.0f} BFS/s, p50 {st.p50_ms:.2f} ms, "
                f"p99 {st.p99_ms:.2f} ms, mean batch {st.mean_batch_size:.1f}")
        out["device_bytes"] = srv.stats().device_bytes
    finally:
        srv.stop()
    return out


def workload_config(args):
    mode = " ".join(x for x, on in (("-A", args.auto_tune), ("-C", args.corebfs),
                                    ("group reordering", args.group_reorder)) if on) or "plain"
    return {"workload": f"Graph500 Kronecker SCALE {args.scale} edgefactor {args.edgefactor} "
                        f"(A,B,C=.57,.19,.19, seeds 2/3), {args.roots} roots, single-source "
                        f"direction-optimizing BFS, {mode}",
            "auto_tune": bool(args.auto_tune),
            "scale": args.scale, "edgefactor": args.edgefactor, "roots": args.roots,
            "corebfs": bool(args.corebfs), "group_reorder": bool(args.group_reorder),
            "alpha": args.alpha, "beta": args.beta,
            "alpha_beta_before_engine_tuner": getattr(args, "alpha_beta_given", None),
            "l2": "inputs larger than L2 (device CSR of tens of GB, pred re-initialised "
                  "every search)",
            "parallelism": "replicas"}


def host_facts():
    """Cores, CPU model and memory of this host (the CPU reference's machine)."""
    model, mem_gb = None, None
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemTotal"):
                mem_gb = int(ln.split()[1]) / 1e6
                break
    except OSError:
        pass
    return {"cores": os.cpu_count(), "cpu": model, "mem_gb": mem_gb}


def run_reference(args, rank, world, dist):
    """The reference arm: the reference's own CPU BFS, i.e. mpi/main.cc with
    its stock BfsBase compiled unchanged against the single-rank MPI runtime
    (oracle/_ref/ref_runnable[_group], built by oracle/ref/Makefile), run as
    `mpiexec -n 1 runnable SCALE [-A] [-C] -n K -v 1` on all host cores.  No
    library of this repository is loaded in the process that runs it.

    SCALE is --ref-scale (default 22), not the GPU arm's 28: the reference
    keeps the edge lists and a 64-bit edge array in host memory (about
    225 GB at SCALE 28, more than this host's 196 GB), and its single-process
    CoreBFS construction takes 213 s at SCALE 22 and 861 s at SCALE 24 on the
    16 host cores, about an hour at SCALE 26.  The options are the GPU arm's
    (-A tuner, -C CoreBFS, group reordering).  Warm-up: W extra roots whose
    searches are dropped; value = harmonic-mean TEPS of the next K roots from
    the reference's own per-root "Time for BFS" and traversed-edge lines."""
    if rank != 0:
        return
    import re

    scale = args.ref_scale
    exe = os.path.join(ROOT, "oracle", "_ref",
                       "ref_runnable_group" if args.group_reorder else "ref_runnable")
    if not os.access(exe, os.X_OK):
        raise SystemExit(f"{exe} missing: build it with `make -C oracle/ref` where the "
                         "reference tree is")
    nroots = min(64, args.warmup + args.steps)
    cmd = [exe, str(scale), "-e", str(args.edgefactor), "-n", str(nroots), "-v", "1",
           "-r", str(args.root_seed)]
    cmd += (["-A"] if args.auto_tune else []) + (["-C"] if args.corebfs else [])
    if not args.auto_tune:
        cmd += ["-a", str(args.alpha), "-b", str(args.beta)]
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    t0 = time.time()
    log("reference: " + " ".join(os.path.relpath(c, ROOT) if c == exe else c for c in cmd))
    p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=args.ref_timeout)
    out = p.stdout + "\n" + p.stderr
    if p.returncode != 0 or "No results printed for invalid run" in out:
        raise SystemExit(f"reference run failed (rc {p.returncode}):\n{out[-3000:]}")
    times = {int(m.group(1)): float(m.group(2))
             for m in re.finditer(r"Time for BFS (\d+) is ([0-9.eE+-]+)", out)}
    # traversed-edge lines carry no index; they follow the roots in order
    counts = [int(m.group(1)) for m in re.finditer(r"Number of traversed edges is (\d+)", out)]
    idx = sorted(times)
    if len(idx) != nroots or len(counts) != nroots:
        raise SystemExit(f"reference output has {len(idx)} timed searches, {len(counts)} edge "
                         f"counts, expected {nroots}")
    keep = idx[args.warmup:] if nroots > args.warmup else idx
    t = [times[i] for i in keep]
    used = [counts[idx.index(i)] for i in keep]
    value = harmonic_teps(used, t) / 1e9

    def field(name):
        m = re.search(r"^%s:\s+(\S+)" % name, out, re.M)
        return float(m.group(1)) if m else None

    cfg = {
        "workload": f"Graph500 Kronecker SCALE {scale} edgefactor {args.edgefactor} "
                    f"(A,B,C=.57,.19,.19, seeds 2/3), {len(keep)} roots, the reference's own "
                    "single-source direction-optimizing BFS on the host CPU, "
                    + " ".join(x for x, on in (("-A", args.auto_tune), ("-C", args.corebfs),
                                               ("group reordering", args.group_reorder)) if on),
        "auto_tune": bool(args.auto_tune), "scale": scale, "edgefactor": args.edgefactor,
        "roots": len(keep), "corebfs": bool(args.corebfs),
        "group_reorder": bool(args.group_reorder),
        "alpha": field("alpha"), "beta": field("beta"),
        "gpu_arm_scale": args.scale,
        "why_not_gpu_arm_scale": "the reference needs about 225 GB of host memory at SCALE 28 "
                                 "(this host has %.0f GB) and about an hour of single-process "
                                 "CoreBFS construction at SCALE 26" % (host_facts()["mem_gb"] or 0),
        "construction_s": field("construction_time"),
        "host": host_facts(),
        "parallelism": "one process, OpenMP on all host cores (mpiexec -n 1)",
    }
    sample = (f"{len(keep)} searches at SCALE {scale} (after {nroots - len(keep)} warm-up "
              f"searches) by the reference's mpi/main.cc + BfsBase, compiled unchanged "
              f"(GNU3 flags, single-rank MPI runtime), {time.time() - t0:.0f} s in all")
    line = {
        "impl": "reference",
        "metric": f"harmonic-mean GTEPS, SCALE {args.scale}; 64-root batched BFS/s + p99 vs 1-root",
        "value": value, "unit": "GTEPS", "n_gpus": world, "steps": len(keep),
        "warmup": nroots - len(keep), "ms_per_step": 1e3 * float(np.mean(t)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (Graph500 Kronecker generator, seeds 2/3)",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local, dist = dist_setup()
    if args.impl == "reference":
        run_reference(args, rank, world, dist)
        if dist is not None:
            dist.destroy_process_group()
        return
    import torch
    import b200bfs

    torch.cuda.set_device(local)
    t0 = time.time()
    eng = b200bfs.Engine(local)
    eng.generate_graph(args.scale, args.edgefactor, flags=build_flags(args))
    t_build = time.time() - t0
    eng.prepare(args.edgefactor, args.alpha, args.beta)
    info = eng.info()
    log(f"[rank {rank}] graph: SCALE {info.scale}, {info.num_global_verts} vertices, "
        f"{info.num_global_edges} directed edges, built in {t_build:.1f}s, "
        f"{info.device_bytes / 1e9:.1f} GB on device")
    roots, nedge, cold_ms = pick_roots(eng, args)
    log(f"[rank {rank}] roots validated; nedge {int(nedge.min())}..{int(nedge.max())}; "
        f"first search after prepare {cold_ms:.3f} ms")
    if args.auto_tune:
        t0 = time.time()
        args.alpha, args.beta, _ = eng.auto_tune(roots, nedge, args.edgefactor, args.alpha,
                                                 args.beta)
        log(f"[rank {rank}] -A tuning: alpha {args.alpha:.4g}, beta {args.beta:.4g} "
            f"({time.time() - t0:.1f}s)")
    for kv in args.engine_option:
        name, value = kv.split("=", 1)
        eng.set_option(name, int(value))
    tuner = None
    if args.tune_engine:
        t0 = time.time()
        what = b200bfs.TUNE_FORMS | b200bfs.TUNE_BATCH_ALPHA
        if args.tune_switch:
            what |= b200bfs.TUNE_SWITCH
        tuner = eng.tune_engine(roots, args.edgefactor, args.alpha, args.beta, what).as_dict()
        if args.tune_switch:
            args.alpha_beta_given = [args.alpha, args.beta]
            args.alpha, args.beta = tuner["alpha"], tuner["beta"]
        log(f"[rank {rank}] engine tuner: {tuner} ({time.time() - t0:.1f}s)")

    stream = torch.cuda.ExternalStream(eng.stream())
    order = [i % len(roots) for i in range(args.warmup + args.steps)]
    for i in order[: args.warmup]:
        eng.run(int(roots[i]), args.edgefactor, args.alpha, args.beta)

    # ---- timed region: device-resident graph ----
    clocks = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    stats = []
    torch.cuda.nvtx.range_push("bench_timed")
    for k, i in enumerate(order[args.warmup:]):
        ev[k][0].record(stream)
        eng.run(int(roots[i]), args.edgefactor, args.alpha, args.beta)
        ev[k][1].record(stream)
        stats.append(eng.run_stats())
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    times = [a.elapsed_time(b) / 1e3 for a, b in ev]
    used = [nedge[i] for i in order[args.warmup:]]
    if dist is not None:
        dist.barrier()
    total = barrier_max(dist, sum(times))
    local_teps = harmonic_teps(used, times)
    # all replicas process the same roots: whole-job rate = sum over ranks at
    # the slowest rank's time
    value = barrier_sum(dist, local_teps * sum(times)) / total / 1e9

    # ---- e2e through the C ABI: search + pred to pinned host memory ----
    pinned = torch.empty(info.pred_size, dtype=torch.int64, pin_memory=True)
    pinned_np = pinned.numpy()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    torch.cuda.synchronize()
    for k, i in enumerate(order[args.warmup:]):
        ev2[k][0].record(stream)
        eng.run(int(roots[i]), args.edgefactor, args.alpha, args.beta)
        eng.get_pred(pinned_np)
        ev2[k][1].record(stream)
    torch.cuda.synchronize()
    times2 = [a.elapsed_time(b) / 1e3 for a, b in ev2]
    # clocks sampled from the start of the device-timed searches to the end
    # of the end-to-end ones (the device-timed region alone is shorter than
    # the sampling interval)
    clk = clocks.stop()
    total2 = barrier_max(dist, sum(times2))
    e2e = barrier_sum(dist, harmonic_teps(used, times2) * sum(times2)) / total2 / 1e9

    # ---- batched multi-source search on the same graph ----
    batched = batched_leg(eng, roots, nedge, args, stream, dist, times,
                          [st.pred_ms for st in stats])

    # ---- roofline of the dominant kernel ----
    td_ms = sum(s.td_ms for s in stats)
    bu_ms = sum(s.bu_ms for s in stats)
    if bu_ms >= td_ms:
        kname, kms, kbytes = "bu_wide_kernel", bu_ms, sum(s.bu_bytes for s in stats)
        launches = sum(s.num_bu_levels for s in stats)
    else:
        kname, kms, kbytes = "td_expand_kernel", td_ms, sum(s.td_bytes for s in stats)
        launches = sum(s.num_td_levels for s in stats)
    peak, peak_kind = peaks()
    achieved = kbytes / (kms / 1e3) / 1e9 if kms > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                "frac_of_nominal_8000_gbs": achieved / 8000.0,
                "traffic": ncu_traffic(kname),
                "algorithmic_bytes_per_launch": kbytes / max(launches, 1),
                "launches": launches, "share_of_search_time":
                    kms / (1e3 * sum(times)) if times else None,
                "whole_search_algorithmic_gbs":
                    sum(s.algorithmic_bytes for s in stats) / sum(times) / 1e9}
    # every kernel group of the search against the same peak
    pred_ms = sum(s.pred_ms for s in stats)
    kernels = {}
    for name, ms, nbytes in (("bu_wide_kernel", bu_ms, sum(s.bu_bytes for s in stats)),
                             ("td_expand_kernel", td_ms, sum(s.td_bytes for s in stats)),
                             ("assemble_pred_kernel", pred_ms,
                              sum(s.pred_bytes for s in stats))):
        if ms > 0:
            gbs = nbytes / (ms / 1e3) / 1e9
            kernels[name] = {"ms_per_search": ms / len(stats), "achieved_gbs": gbs,
                             "frac": gbs / peak, "frac_of_nominal_8000_gbs": gbs / 8000.0,
                             "share_of_search_time": ms / (1e3 * sum(times)),
                             "traffic": ncu_traffic(name)}
    # The top-down levels are random 4-byte probes of the visited bitmap (one
    # per adjacency entry) and ORs (one per claim): the device's rate of such
    # accesses into a buffer the size of that bitmap, measured here, bounds
    # them where the HBM bandwidth does not.  ceiling_ms counts the probes
    # only, so the fraction is a lower bound.
    if "td_expand_kernel" in kernels:
        kernels["td_expand_kernel"]["random_access"] = td_random_access(
            eng, info, stats, td_ms, stream)

    line = {
        "metric": f"harmonic-mean GTEPS, SCALE {args.scale}; 64-root batched BFS/s + p99 vs 1-root",
        "value": value, "unit": "GTEPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (Graph500 Kronecker generator on the device, seeds 2/3)",
        "config": workload_config(args),
        "e2e": {"value": e2e, "unit": "GTEPS", "h2d_bytes_per_step": 8,
                "d2h_bytes_per_step": 8 * info.pred_size},
        "roofline": roofline,
        "kernels": kernels,
        "clocks": clk,
        "gpu_launches": int(barrier_sum(dist, sum(s.kernel_launches for s in stats))),
        "batched": batched,
        "engine_tuner": tuner,
        "search": {"edges_scanned_per_input_edge":
                       float(np.mean([(s.edges_scanned_td + s.edges_scanned_bu) for s in stats]))
                       / (info.num_input_edges or 1),
                   "levels": int(np.median([s.levels for s in stats])),
                   "td_ms": td_ms / args.steps, "bu_ms": bu_ms / args.steps,
                   "pred_ms": pred_ms / args.steps,
                   "first_search_after_prepare_ms": cold_ms,
                   "build_s": t_build},
    }
    eng.end()
    eng.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_leg(args, local, roots, nedge)
    if world == 1 and not args.no_serve:
        line["serving"] = serving_leg(args, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
