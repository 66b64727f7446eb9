"""Benchmark of the traversal hot path: SSSP (delta-stepping) and BFS (direction-optimising) GTEPS on B200.

Workload (default): RMAT scale 23 (V = 8,388,608), edge factor 32 (268,435,456 directed edges before the
self-loop drop), a/b/c/d = 57/19/19/5, fp32 weights rand_r/RAND_MAX, seed 1, self-loops dropped; 64 seeded
sources of nonzero out-degree.  One step = BFS (Beamer alpha 15 / beta 18) from each of the 64 sources plus
SSSP (delta-stepping, delta 0.1) from each of them, the 128 queries run as one batched persistent launch
(teams of CTAs, one query each at a time; shape autotuned outside the timed region).  TEPS = edges in the
graph / traversal time (the reference's convention), summed over traversals.  The graph (4.4 GB of CSR, CSC
and in-edge weights) is larger than the 126 MB L2, so no flush runs between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--scale S] [--ef F]

Under torchrun each rank runs an independent replica on its own GPU (the path has no data-path exchange):
weak scaling, value = traversals of all ranks x E / max-over-ranks time.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "parallel-task1_b200")
sys.path.insert(0, PKG)

METRIC = "SSSP/BFS GTEPS on 1 B200, learned vs plain schedule, bit-exact"
ABCD = (57, 19, 19, 5)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=23)
    ap.add_argument("--ef", type=int, default=32)
    ap.add_argument("--sources", type=int, default=64)
    ap.add_argument("--delta", type=float, default=0.1)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-parts", type=int, default=1, help="launches the e2e step is cut into")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip the reference's own GPU path")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched many-graph measurement")
    ap.add_argument("--batched-only", action="store_true", help="run only the batched many-graph measurement")
    ap.add_argument("--cpu-sample-s", type=float, default=20.0, help="target seconds of CPU baseline work")
    ap.add_argument("--save-tune-table", default=None,
                    help="write the table of autotuned launch shapes here at the end (a file for weights/)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_name(a):
    """The workload both arms solve: the graph, the sources and the two queries per source.  How each arm
    computes them (delta-stepping or Bellman-Ford; Beamer's switch or a level-synchronous top-down sweep) is
    in the line's `implementation`; the distances and reachability are the same bits."""
    return (f"RMAT s{a.scale} ef{a.ef} a/b/c/d 57/19/19/5 seed {a.seed} loops dropped; {a.sources} sources; "
            f"BFS + SSSP (delta {a.delta}) from each source")


def bench_config(a, V, E, world):
    """config of the JSON line; identical keys and values in both arms for the same arguments."""
    return {"workload": workload_name(a), "scale": a.scale, "edge_factor": a.ef, "vertices": V, "edges": E,
            "sources": a.sources, "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"}


def host_cpu():
    """CPU model, physical cores and logical CPUs of this host."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        import psutil

        phys = psutil.cpu_count(logical=False)
    except Exception:
        phys = None
    return {"cpu_model": model, "physical_cores": phys, "logical_cpus": os.cpu_count()}


def pick_sources(deg, n, seed):
    """n distinct seeded sources among vertices of nonzero out-degree (sorted)."""
    rng = np.random.default_rng(seed)
    cand = np.flatnonzero(deg > 0)
    return np.sort(rng.choice(cand, size=min(n, len(cand)), replace=False)).astype(np.int32)


def rank_sources(deg, n, seed, rank):
    """Replica r of a weak-scaling run traverses its own seeded source set."""
    return pick_sources(deg, n, seed + rank)


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Max of a per-rank time over the process group (the slowest replica sets the job time)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gteps(traversals_per_rank: int, edges: int, world: int, seconds_max: float) -> float:
    """Whole-job GTEPS: every rank's traversals x E over the max-over-ranks time."""
    return world * traversals_per_rank * edges / seconds_max / 1e9


# --------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of the GPU clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.seek(0)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = max(smax, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str, queries: int = 1, workload: str = ""):
    """DRAM bytes per launch of `kernel` on `workload` (e.g. rmat_s23_ef32) from the committed ncu summary
    (profiles/traffic.txt), if any.  An entry with bytes_per_query (a capture of fewer queries than the bench's
    launch, on the same graph) is scaled to `queries`; an entry for another workload does not count."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            kv = dict(x.split("=", 1) for x in line.split() if "=" in x)
            if kv.get("kernel") != kernel or kv.get("workload", workload) != workload:
                continue
            if "bytes_per_launch" in kv:
                return float(kv["bytes_per_launch"])
            if "bytes_per_query" in kv:
                return float(kv["bytes_per_query"]) * queries
    return None


# -------------------------------------------------------------- CPU side
class CpuReference:
    """The reference's own CPU path (oracle/_ref) on the same workload, timed on bounded samples.

    The graph is the same seeded RMAT (the oracle's generator restates the reference's and is
    bit-identical to the device generator); the EL and CSR containers are built once, untimed.  SSSP is
    the reference's cpu_bellman_ford, BFS its cpu_parallel_bfs, both with every host core.
    """

    def __init__(self, a, threads=None):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        if not O.ref_available():
            raise RuntimeError("oracle/_ref/libtrav_ref.so is missing")
        self.O = O
        self.cores = threads or os.cpu_count() or 1
        s, d, w = O.rmat(a.scale, a.ef, ABCD, seed=a.seed, drop_self_loops=True, threads=self.cores)
        V = 1 << a.scale
        self.E = len(s)
        self.sources = pick_sources(np.bincount(s, minlength=V), a.sources, a.seed)
        self.gel = O.RefGraph.edges_list(V, s, d, w)
        off, adj, wt = O.csr(V, s, d, w)
        del s, d, w
        self.gcsr = O.RefGraph.csr(V, off, adj, wt)
        self.next = 0

    def sample(self, seconds, check=None):
        """GTEPS of the GPU step's mix (one BFS + one SSSP per source) over about `seconds` of work.  With
        `check`, check(source_index, reached, dist) is called after each source's two calls, outside their
        timing brackets, with the reference's own results."""
        O = self.O
        t_sssp, t_bfs = [], []
        start = time.perf_counter()
        while not t_sssp or (time.perf_counter() - start) < seconds:
            k = self.next % len(self.sources)
            src = int(self.sources[k])
            self.next += 1
            t0 = O.ref().ref_wtime()
            reached = self.gcsr.parallel_bfs(src, threads=self.cores)
            t_bfs.append(O.ref().ref_wtime() - t0)
            t0 = O.ref().ref_wtime()
            dist = self.gel.bellman_ford(src, threads=self.cores)
            t_sssp.append(O.ref().ref_wtime() - t0)
            if check is not None:
                check(k, reached, dist)
        per_source = statistics.mean(t_bfs) + statistics.mean(t_sssp)
        desc = (f"{len(t_bfs)} cpu_parallel_bfs + {len(t_sssp)} cpu_bellman_ford calls of the reference "
                f"(oracle/_ref) on the same graph and sources with {self.cores} threads; GTEPS = 2E / (mean BFS + "
                f"mean SSSP time); mean BFS {statistics.mean(t_bfs):.3f} s, mean SSSP {statistics.mean(t_sssp):.3f} s")
        return 2 * self.E / per_source / 1e9, desc

    def free(self):
        self.gel.free()
        self.gcsr.free()


def cpu_reference_run(a, seconds, levels=None, dist=None):
    """The CPU baseline leg: the reference's own path timed on a bounded sample.  With the GPU step's results
    (levels[k], dist[k] of source k, original ids), every sampled source's reference results are compared with
    them bit for bit: distances exactly, reachability as level >= 0; the returned parity record says how many
    sources were compared and whether all were equal."""
    ref = CpuReference(a)
    parity = {"sources": 0, "equal": True, "compared": "cpu_bellman_ford distance bits and cpu_parallel_bfs "
                                                      "reachability of the same sources against the GPU step"}

    def check(k, reached, d):
        if levels is None:
            return
        same = (np.array_equal(d.view(np.uint32), dist[k].view(np.uint32))
                and np.array_equal(reached.astype(bool), levels[k] >= 0))
        parity["sources"] += 1
        parity["equal"] = parity["equal"] and bool(same)

    try:
        v, desc = ref.sample(seconds, check=check if levels is not None else None)
        return v, desc, ref.cores, ref.E, (parity if levels is not None else None)
    finally:
        ref.free()


def reference_gpu_run(a, cap_s: float = 90.0):
    """The reference's own GPU path (its bellman_ford.cu and bfs.cu built unchanged for sm_100a, oracle/_ref) on
    the same graph and sources: per source, bfs_wrapper then init_distances_wrapper + bellman_ford_wrapper on an
    edge list resident in device memory, timed as the reference times them (host clock around the wrappers,
    uploads excluded).  Stops after cap_s seconds of wrapper time and reports the sources it finished."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if not O.refgpu_available():
        return {"unavailable": "oracle/_ref/libtrav_refgpu.so is not built (needs the reference sources)"}
    V = 1 << a.scale
    s, d, w = O.rmat(a.scale, a.ef, ABCD, seed=a.seed, drop_self_loops=True, threads=os.cpu_count() or 1)
    E = len(s)
    sources = pick_sources(np.bincount(s, minlength=V), a.sources, a.seed)
    L = O.refgpu()
    if L.refgpu_upload(V, E, s, d, w) != 0:
        return {"unavailable": "device allocation for the reference's edge list failed"}
    del s, d, w
    dist = np.empty(V, np.float32)
    vis = np.empty(V, np.uint8)
    t_bfs, t_sssp = [], []
    try:
        with O.quiet_stdout():
            for src in sources.tolist():
                tb = L.refgpu_bfs(src, vis)
                ts = L.refgpu_sssp(src, dist)
                if tb < 0 or ts < 0:
                    break
                t_bfs.append(tb)
                t_sssp.append(ts)
                if sum(t_bfs) + sum(t_sssp) > cap_s:
                    break
    finally:
        L.refgpu_free()
    if not t_bfs:
        return {"unavailable": "the reference's GPU wrappers failed on this workload"}
    total = sum(t_bfs) + sum(t_sssp)
    return {"gteps": 2 * len(t_bfs) * E / total / 1e9, "sources": len(t_bfs), "ms_per_step_64": total / len(t_bfs) * 64e3,
            "mean_bfs_ms": 1e3 * statistics.mean(t_bfs), "mean_sssp_ms": 1e3 * statistics.mean(t_sssp),
            "what": "the reference's bfs_wrapper + init_distances_wrapper/bellman_ford_wrapper (its bellman_ford.cu "
                    "and bfs.cu built unchanged for sm_100a) per source on a resident edge list; host clock around "
                    "the wrappers as the reference times them; GTEPS = 2E x sources / total time"}


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    ref = CpuReference(a)
    E, cores = ref.E, ref.cores
    t_steps = []
    desc = None
    budget = max(3.0, 90.0 / max(a.steps + a.warmup, 1))
    for k in range(a.warmup + a.steps):
        v, desc = ref.sample(budget)
        if k >= a.warmup:
            t_steps.append(v)
    ref.free()
    value = statistics.median(t_steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 2 * E / value / 1e6, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded RMAT generated here)",
        "config": bench_config(a, 1 << a.scale, E, a.gpus),
        "implementation": ("the reference's own CPU path (oracle/_ref, compiled from its sources): "
                           "cpu_parallel_bfs (level-synchronous top-down, bool reachability) and cpu_bellman_ford "
                           "(edge-list sweeps to the fixpoint) per source, all host threads"),
        "cpu_baseline": dict({"value": value, "unit": "GTEPS", "cores": cores, "kind": "reference",
                              "sample": desc}, **host_cpu()),
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------- GPU side
def run_ours(a):
    import torch
    import torch.distributed as dist

    import pytrav as T

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if a.batched_only:
        if rank == 0:
            print(json.dumps({"batched": batched_workload(a.seed)}), flush=True)
        return
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)

    t0 = time.perf_counter()
    g = T.Graph.rmat(a.scale, a.ef, ABCD, seed=a.seed, drop_self_loops=True)
    torch.cuda.synchronize()
    ingest_s = time.perf_counter() - t0
    V, E = g.V, g.E
    deg = g.out_degrees()
    sources = rank_sources(deg, a.sources, a.seed, rank)
    n = len(sources)

    stream = torch.cuda.current_stream()
    g.set_stream(stream)
    lv_dev = torch.empty((n, V), dtype=torch.int32, device=dev)
    di_dev = torch.empty((n, V), dtype=torch.float32, device=dev)

    from pytrav import learn

    have_learned = learn.install(g, delta=a.delta)  # trained schedule networks shipped in parallel-task1_b200/weights
    schedules = ([T.SCHEDULE_LEARNED] if have_learned else []) + [T.SCHEDULE_PLAIN]
    primary = schedules[0]
    names = {T.SCHEDULE_PLAIN: "plain", T.SCHEDULE_LEARNED: "learned"}

    # One step = BFS and SSSP from every source.  The 2n queries run concurrently in one batched persistent
    # launch (trav_batch_run): teams of CTAs each run one query at a time, so the latency-bound tails of one
    # query overlap the work of others.  The launch shape is autotuned once per schedule, outside the timed region.
    import ctypes

    batch = T.Batch([g])
    # launch shapes tuned on earlier runs (parallel-task1_b200/weights/batch_shapes.txt): a kind of batch found
    # there is not re-tuned; anything else is tuned once and added to this process's table
    if os.path.exists(T.TUNE_TABLE):
        T.tune_table_load()
    queries = {sched: [(0, 0, int(s), 0.0, sched, lv_dev[i]) for i, s in enumerate(sources)]
               + [(0, 1, int(s), a.delta, sched, di_dev[i]) for i, s in enumerate(sources)]
               for sched in schedules}

    def step(sched, record):
        ms = batch.run(queries[sched])
        if record is not None:
            record.append(ms)

    # Each schedule: algorithmic bytes per traversal measured once per source outside the timed region (the
    # SSSP count is schedule-independent; the BFS count follows the direction trace, which is deterministic),
    # the shape autotuned, W warm-up steps, then K timed steps bracketed by a barrier and a device
    # synchronisation; the step time is the device time of its launch (CUDA events around it).
    runs = {}
    clk = None
    for sched in schedules:
        bfs_bytes, sssp_bytes = [], []
        for s in sources:
            g.bfs([s], out=lv_dev[:1], schedule=sched)
            bfs_bytes.append(g.last_stats().algorithmic_bytes)
            g.sssp([s], out=di_dev[:1], delta=a.delta, schedule=sched)
            sssp_bytes.append(g.last_stats().algorithmic_bytes)
        shape = batch.autotune(queries[sched], reps=0)
        for _ in range(a.warmup):
            step(sched, None)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local) if sched == primary else None
        if clocks:
            clocks.start()
        rec = []
        for _ in range(a.steps):
            step(sched, rec)
        torch.cuda.synchronize()
        if clocks:
            clk = clocks.stop()
        if world > 1:
            dist.barrier()
        ms_max = max_over_ranks(sum(rec), world, dev)
        runs[sched] = dict(ms=ms_max, rec=rec, bfs_bytes=bfs_bytes, sssp_bytes=sssp_bytes, shape=shape,
                           lv=lv_dev.cpu().numpy(), di=di_dev.cpu().numpy())
    traversals = 2 * n * a.steps
    value = job_gteps(traversals, E, world, runs[primary]["ms"] / 1e3)
    if len(runs) == 2:  # both schedules must give the same bits
        assert np.array_equal(runs[0]["lv"], runs[1]["lv"])
        assert np.array_equal(runs[0]["di"].view(np.uint32), runs[1]["di"].view(np.uint32))

    # the same step as one persistent launch per query (the single-query API), for comparison
    seq_ms = []
    for rep in range(3):
        g.bfs(sources, out=lv_dev, schedule=primary)
        t = float(np.sum(g.last_batch_ms()))
        g.sssp(sources, out=di_dev, delta=a.delta, schedule=primary)
        t += float(np.sum(g.last_batch_ms()))
        if rep:
            seq_ms.append(t)
    seq_ms = min(seq_ms)
    assert np.array_equal(runs[primary]["lv"], lv_dev.cpu().numpy())
    assert np.array_equal(runs[primary]["di"].view(np.uint32), di_dev.cpu().numpy().view(np.uint32))

    # e2e through the library's host-output batch call (trav_batch_run_host) with pinned host buffers: per step,
    # the query descriptors (source ids inside) go H2D in the call and every level / distance array comes back
    # D2H into the caller's host memory.  The library runs the 128 queries (each source's SSSP and BFS side by
    # side) in --e2e-parts launches and copies each query's results as soon as its team has written them, while
    # the launch runs on (the cheap queries are spread through the launch so the copies keep pace).  Timed on
    # the host clock.
    lv_host = torch.empty((n, V), dtype=torch.int32).pin_memory()
    di_host = torch.empty((n, V), dtype=torch.float32).pin_memory()
    host_queries = []
    for i, s in enumerate(sources):
        host_queries.append((0, 1, int(s), a.delta, primary, di_host[i]))
        host_queries.append((0, 0, int(s), 0.0, primary, lv_host[i]))

    def e2e_step():
        batch.run_host(host_queries, parts=a.e2e_parts)

    for _ in range(max(1, min(a.warmup, 2))):
        e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    h0 = time.perf_counter()
    for _ in range(a.steps):
        e2e_step()
    h1 = time.perf_counter()
    e2e_value = job_gteps(traversals, E, world, max_over_ranks(h1 - h0, world, dev))
    h2d = len(queries[primary]) * ctypes.sizeof(T.Query)

    # parity spot check of the timed outputs against the host copies (same kernels, same inputs)
    assert np.array_equal(runs[primary]["lv"], lv_host.numpy())
    assert np.array_equal(runs[primary]["di"].view(np.uint32), di_host.numpy().view(np.uint32))
    batch.close()

    # roofline of the timed kernel: all queries' algorithmic bytes over the launch's device time
    rec = runs[primary]["rec"]
    mean_ms = statistics.mean(rec)
    launch_bytes = float(sum(runs[primary]["sssp_bytes"]) + sum(runs[primary]["bfs_bytes"]))
    achieved = launch_bytes / (mean_ms / 1e3) / 1e9
    peak, peak_src = measured_peaks()
    kname = "batch_persistent"
    traffic = ncu_traffic(kname, queries=len(queries[primary]), workload=f"rmat_s{a.scale}_ef{a.ef}")

    if rank == 0:
        per = {names[k]: {"gteps": job_gteps(traversals, E, world, r["ms"] / 1e3), "ms_per_step": r["ms"] / a.steps,
                          "shape": {"team_ctas": r["shape"][0], "small_deg": r["shape"][1], "item": r["shape"][2]}}
               for k, r in runs.items()}
        line = {
            "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": runs[primary]["ms"] / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded RMAT generated on the device)",
            "config": bench_config(a, V, E, world),
            "implementation": (f"BFS direction-optimising (Beamer alpha 15 / beta 18 or the learned switch) and "
                               f"SSSP delta-stepping (delta {a.delta}, light/heavy edges, pull rounds); each step's "
                               f"2n queries in one batched persistent launch (autotuned teams)"),
            "schedule": names[primary],
            "schedules": per,
            "sequential_launches": {"gteps": job_gteps(2 * n, E, 1, seq_ms / 1e3), "ms_per_step": seq_ms,
                                    "note": "the same step as one persistent launch per query, primary schedule"},
            "learned_over_plain": (per["learned"]["gteps"] / per["plain"]["gteps"]) if "learned" in per else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kname,
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_launch": launch_bytes, "mean_launch_ms": mean_ms,
                         "queries_per_launch": len(queries[primary])},
            "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": 2 * 4 * n * V,
                    "timing": f"host clock around trav_batch_run_host (host output arrays; {a.e2e_parts} "
                              f"launch(es); each query's results copied back as soon as its team has written "
                              f"them, while the launch runs on; cheap queries spread through the launch so the "
                              f"copies keep pace)"},
            "gpu_launches": a.steps,
            "ingest_s": ingest_s,
            "clocks": clk,
        }
        if not a.no_batched and world == 1:
            line["batched"] = batched_workload(a.seed)
        if not a.no_cpu_baseline and world == 1:
            try:
                v, desc, cores, _, parity = cpu_reference_run(a, a.cpu_sample_s, levels=runs[primary]["lv"],
                                                              dist=runs[primary]["di"])
                line["cpu_baseline"] = dict({"value": v, "unit": "GTEPS", "cores": cores, "kind": "reference",
                                             "sample": desc}, **host_cpu())
                line["parity"] = parity
            except Exception as ex:  # the baseline is reported, never required for the GPU number
                line["cpu_baseline"] = dict({"value": None, "unit": "GTEPS", "cores": os.cpu_count(),
                                             "kind": "reference", "sample": f"not run: {ex}"}, **host_cpu())
        if not a.no_reference_gpu and world == 1:
            try:
                line["reference_gpu"] = reference_gpu_run(a)
            except Exception as ex:  # a reported baseline, never required for the GPU number
                line["reference_gpu"] = {"unavailable": f"not run: {ex}"}
        print(json.dumps(line), flush=True)
        if a.save_tune_table:
            T.tune_table_save(a.save_tune_table)
    g.free()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def batched_workload(seed: int) -> dict:
    """The batched workload: 64 seeded RMAT graphs (scale 10-18 and edge factor 8-32 drawn uniformly, the
    workload's a/b/c/d, weights rand_r/RAND_MAX) with 8 sources each, 512 queries alternating BFS and SSSP
    (delta 0.1), in one persistent launch with the autotuned shape, against one launch per query through the
    single-query API.  Results of the two must be identical."""
    import torch

    import pytrav as T

    rng = np.random.default_rng(seed + 1000)
    graphs = []
    for i in range(64):
        scale, ef = int(rng.integers(10, 19)), int(rng.integers(8, 33))
        graphs.append(T.Graph.rmat(scale, ef, ABCD, seed=seed + 100 + i, drop_self_loops=True))
    queries = []
    for gi, g in enumerate(graphs):
        deg = g.out_degrees()
        for k, s in enumerate(rng.choice(np.flatnonzero(deg > 0), 8, replace=False)):
            kind = k % 2
            out = torch.empty(g.V, dtype=torch.int32 if kind == 0 else torch.float32, device="cuda")
            queries.append((gi, kind, int(s), 0.1, T.SCHEDULE_PLAIN, out))
    edges = sum(graphs[q[0]].E for q in queries)
    single_ms = 0.0
    for _ in range(2):  # the second pass is timed (device events of each launch)
        single_ms = 0.0
        for gi, kind, s, delta, _, out in queries:
            g = graphs[gi]
            if kind == 0:
                g.bfs([s], out=out.view(1, -1))
            else:
                g.sssp([s], out=out.view(1, -1), delta=delta)
            single_ms += g.last_stats().kernel_ms
    ref = [q[5].clone() for q in queries]
    b = T.Batch(graphs)
    t0 = time.perf_counter()
    if os.path.exists(T.TUNE_TABLE):
        T.tune_table_load()
    shape = b.autotune(queries, reps=0)
    tune_s = time.perf_counter() - t0
    for q in queries:
        q[5].fill_(7)
    runs = [b.run(queries) for _ in range(5)]
    same = all(torch.equal(q[5], r) for q, r in zip(queries, ref))
    assert same, "batched results differ from the single-query results"
    ms = statistics.median(runs)
    b.close()
    for g in graphs:
        g.free()
    return {"workload": "64 RMAT graphs (scale 10-18, edge factor 8-32), 8 sources each: 512 queries, "
                        "BFS and SSSP (delta 0.1) alternating", "queries": len(queries), "edges_traversed": edges,
            "ms": ms, "gteps": edges / (ms / 1e3) / 1e9, "shape": {"team_ctas": shape[0], "small_deg": shape[1],
                                                                 "item": shape[2]},
            "autotune_s": tune_s, "single_launch_ms": single_ms,
            "single_launch_gteps": edges / (single_ms / 1e3) / 1e9, "speedup_over_single_launches": single_ms / ms,
            "identical_results": same, "timing": "device events around the one launch (median of 5)"}


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
