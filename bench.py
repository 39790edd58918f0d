"""Benchmark of the subgraph-matching hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (plain method, larger graph): an R-MAT data graph (scale 20 =
1,048,576 vertices, a=.57 b=c=.19, edge factor 8, ~8.0M undirected edges
after symmetrising and dedup) with 32 uniform labels, and 200 random-walk
queries (100 of 12 and 100 of 16 vertices, half sparse / half dense), CFL
filter + CFL order, embedding counts capped at 1e9, one query per launch
sequence. Synthetic data generated from fixed seeds (no dataset download).

One step = the 200 queries through the plain path. `value` is queries/s
from the device time of the launches (CUDA events on the library's stream,
graph resident in HBM); `e2e` is the same through the C ABI call psm_match
with host query buffers, host->device descriptor copies (through the
context's pinned staging buffer) and device->host result reads inside the
wall-clock timed region. The data graph (72 MB) fits in L2, so L2 is flushed
(256 MiB write) before every timed step. With N GPUs each rank runs the whole
workload on its own replica of the graph (replicas only, weak scaling); times
are the max over ranks.

At N=1 the same line also carries the other workloads of the path:
`batched_mixed` (2,000 queries of 4-32 vertices on the same graph, batched vs
plain, counts equal), `serve` (R-MAT scale 24, a 50,000-request Poisson
stream at 50/80/95 % of saturation, p50/p99) and `cpu_baseline` (the
reference binary on the host cores, whole queries, counts compared).

--impl reference times the reference's own CPU implementation (the
SubgraphMatching.out binary built from the reference sources by
oracle/Makefile) on the host cores: one step is one whole query of the same
workload run to its end (count = min(total, 1e9), Overtime: 0), and the steps
run as concurrent reference processes, one per host thread.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "queries/sec (plain GPU path, CFL_CFL_EXPLORE, cap 1e9)"
WORKLOAD = "plain_rmat_s20"
REF_BIN = ROOT / "oracle" / "_ref" / "SubgraphMatching.out"
# The reference counts a capped query exactly only with one thread per
# process: with more threads every task counts up to the cap on its own
# (EvaluateQuery.cpp:137,152), so a multi-threaded run of a capped query
# overshoots the cap (4.4e9 counted in 30 s on 8 threads) and runs until its
# time limit. The host's threads are therefore used as concurrent one-thread
# processes, one query each; one multi-threaded run is reported beside them.
REF_NOTE = ("whole queries, one reference process per host thread, -threadnums 1 each: a multi-threaded "
            "reference run of a capped query overshoots the cap and runs until its time limit (see 'multithread')")


def enum_traffic():
    """Mean DRAM bytes per enum_kernel launch of this workload, from the ncu
    capture summarised in profiles/ (None if absent)."""
    p = ROOT / "profiles" / "enum_kernel_traffic_plain_rmat_s20.md"
    if p.exists():
        m = re.search(r"traffic_bytes_per_launch: (\d+)", p.read_text())
        if m:
            return int(m.group(1))
    return None


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the
    timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.rows.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_workload(args):
    from psm_benchmark_b200 import gen
    w = gen.plain_rmat(num_queries=args.queries, scale=args.scale)
    if args.only:
        # a subset of the workload's queries (profiling of single launches)
        w.queries = [w.queries[int(i)] for i in args.only.split(",")]
    return w


def workload_config(w, world):
    """The `config` object of both arms (same workload, same keys)."""
    sizes = sorted({q.num_vertices for q in w.queries})
    return {"workload": WORKLOAD, "graph": f"R-MAT scale {int(np.log2(w.graph.num_vertices))}, edge factor 8, "
                                          "32 uniform labels",
            "vertices": w.graph.num_vertices, "edges": w.graph.num_edges, "queries_per_step": len(w.queries),
            "query_sizes": " + ".join(f"{sum(q.num_vertices == k for q in w.queries)} x {k}" for k in sizes),
            "method": w.method, "cap": w.cap, "parallelism": f"replicas x{world}",
            "l2": "flushed (256 MiB write) before every step; 72 MB graph L2-resident within a step"}


# --------------------------------------------------------------- reference --

def ref_available():
    return REF_BIN.exists() and os.access(REF_BIN, os.X_OK)


def run_reference_query(data_txt, qpath, threads, cap, log: Path, time_limit=600):
    """One SubgraphMatching.out run in -QorCandi C mode; returns (Total time,
    #Embeddings, Overtime) from its log block."""
    if log.exists():
        log.unlink()
    cmd = [str(REF_BIN), "-d", data_txt, "-q", qpath, "-threadnums", str(threads),
           "-num", str(cap) if cap else "MAX", "-time_limit", str(int(time_limit)), "-OutputFile", str(log),
           "-QorCandi", "C", "-split", "linear", "-schedule", "busy2idlenostop", "-BackMethods", "CFL_CFL_EXPLORE"]
    subprocess.run(cmd, check=True, capture_output=True, timeout=time_limit + 300)
    text = log.read_text()
    total = float(re.findall(r"Total time \(seconds\): ([0-9.e+-]+)", text)[-1])
    count = int(re.findall(r"#Embeddings: (\d+)", text)[-1])
    over = int(re.findall(r"Overtime: (\d+)", text)[-1])
    return total, count, over


def ref_workers():
    return max(1, os.cpu_count() or 1)


class ReferenceRunner:
    """Writes the workload in the reference's text format once and runs the
    reference binary on its queries, as concurrent one-query processes."""

    def __init__(self, w):
        from psm_benchmark_b200 import gen
        self.tmp = Path(tempfile.mkdtemp(prefix="psmref_"))
        d = self.tmp / "d1" / "d2"
        d.mkdir(parents=True)
        self.data_txt = str(d / "graph.txt")
        gen.write_text(w.graph, self.data_txt)
        qd = self.tmp / "q1" / "q2" / "q3"
        qd.mkdir(parents=True)
        self.qpaths = []
        for i, q in enumerate(w.queries):
            p = qd / f"q{i}.txt"
            q.write_text(p)
            self.qpaths.append(str(p))
        self.cap = w.cap

    def pool(self, indices, workers, threads=1, time_limit=600):
        """Runs the queries `indices` (one process each, `threads` threads per
        process) on `workers` concurrent slots. Returns the runs as
        (query index, slot, total_s, count, overtime), the makespan over
        slots of the reference's own Total time (graph loading excluded, as
        in the reference's log) and the wall time."""
        lock = threading.Lock()
        slots = {}
        runs = []

        def one(i):
            tid = threading.get_ident()
            with lock:
                slot = slots.setdefault(tid, len(slots))
            log = self.tmp / f"log_{slot}.txt"
            t, c, over = run_reference_query(self.data_txt, self.qpaths[i % len(self.qpaths)], threads, self.cap,
                                             log, time_limit)
            with lock:
                runs.append((i, slot, t, c, over))

        t0 = time.time()
        with ThreadPoolExecutor(max_workers=workers) as ex:
            for f in [ex.submit(one, i) for i in indices]:
                f.result()
        wall = time.time() - t0
        per_slot = {}
        for _, slot, t, _, _ in runs:
            per_slot[slot] = per_slot.get(slot, 0.0) + t
        return sorted(runs), max(per_slot.values()), wall


def cpu_info():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def reference_multithread(rr, threads, limit):
    """One run of query 0 with the reference's own multi-threaded engine."""
    t, c, over = run_reference_query(rr.data_txt, rr.qpaths[0], threads, rr.cap, rr.tmp / "log_mt.txt", limit)
    return {"threads": threads, "time_limit_s": limit, "total_s": t, "embeddings": c, "overtime": over,
            "reached_cap": bool(rr.cap and c >= rr.cap), "embeddings_per_s": c / t if t > 0 else None,
            "note": "one query, -threadnums = host threads; a capped query overshoots the cap (tasks count to the "
                    "cap independently, EvaluateQuery.cpp:137,152) and stops only at the time limit"}


def reference_arm(args, world, rank):
    if rank != 0:
        return
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference binary oracle/_ref/SubgraphMatching.out "
                                                              "was not built (reference sources absent at build)"}))
        return
    w = make_workload(args)
    rr = ReferenceRunner(w)
    workers = ref_workers()
    nq = len(w.queries)
    # warm-up: the graph file and the binary into the page cache
    rr.pool([nq - 1 - i for i in range(args.warmup)], workers, time_limit=1)
    runs, makespan, wall = rr.pool(list(range(args.steps)), workers, time_limit=args.ref_limit)
    over = sum(r[4] for r in runs)
    value = len(runs) / makespan
    mt = reference_multithread(rr, workers, args.ref_mt_limit) if args.ref_mt_limit > 0 else None
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": makespan * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": workload_config(w, args.gpus),
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": workers, "kind": "reference",
                             "sample": f"{len(runs)} whole queries (workload queries 0-{len(runs) - 1}), one per step, "
                                       f"on {workers} concurrent one-thread reference processes; value = queries / "
                                       f"makespan of the reference's Total time ({makespan:.1f} s; wall with graph "
                                       f"loading {wall:.1f} s); {over} run(s) hit the time limit; CPU {cpu_info()} "
                                       f"({os.cpu_count()} threads)",
                             "counts": [r[3] for r in runs], "wall_s": wall, "note": REF_NOTE},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if mt is not None:
        line["multithread"] = mt
    print(json.dumps(line))


# -------------------------------------------------------------------- ours --

def flush_l2(buf):
    buf.add_(1)


def scaled_bytes(r, cap):
    """Algorithmic bytes of a query, scaled to the cap when the enumerator
    counted past it before the stop reached every warp: bytes and the
    unclamped count come from the same extended partial embeddings, so
    bytes x cap / count_internal is the work of `cap` embeddings at the
    query's own bytes per embedding."""
    if cap and r.count_internal > cap:
        return r.alg_bytes * cap / r.count_internal
    return float(r.alg_bytes)


def cpu_baseline(w, counts, n):
    """The reference binary on the host cores: n whole queries of the
    workload (queries 0..n-1), concurrent one-thread processes, counts
    compared with this arm's."""
    rr = ReferenceRunner(w)
    runs, makespan, wall = rr.pool(list(range(n)), ref_workers())
    checked = 0
    for i, _, _, c, over in runs:
        if not over:
            if c != counts[i]:
                raise SystemExit(f"reference count {c} differs from ours {counts[i]} (query {i})")
            checked += 1
    return {"value": len(runs) / makespan, "unit": "queries/s", "cores": min(ref_workers(), n), "kind": "reference",
            "sample": f"{len(runs)} whole queries (workload queries 0-{len(runs) - 1}) on {min(ref_workers(), n)} "
                      f"concurrent one-thread reference processes; value = queries / makespan of the reference's "
                      f"Total time ({makespan:.1f} s; wall with graph loading {wall:.1f} s); CPU {cpu_info()} "
                      f"({os.cpu_count()} threads)",
            "reference_counts_checked": checked, "note": REF_NOTE}


def ours_arm(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        # collectives here are seconds apart: a short timeout ends a run whose
        # rank failed instead of leaving the others waiting
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from psm_benchmark_b200 import api
    w = make_workload(args)
    eng = api.Engine(device=local, arena_bytes=args.arena_gb << 30)
    if args.intersect != "BINARY":
        eng.set_batch_tuning(intersect=args.intersect)
    dg = api.DataGraph.from_graph(w.graph)
    flush = torch.empty(256 << 20 >> 2, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def step():
        res = []
        for q in w.queries:
            res.append(api.match(eng, dg, q, w.method, cap=w.cap, time_limit=args.time_limit))
        return res

    for _ in range(args.warmup):
        flush_l2(flush)
        torch.cuda.synchronize()
        step()
    clocks = ClockSampler(local).start()
    barrier()
    dev_ms = 0.0
    enum_ms = 0.0
    alg = 0.0
    lat = []
    h2d = d2h = 0
    counts = None
    internal = 0
    t0 = time.perf_counter()
    for s in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        res = step()
        dev_ms += sum(r.prep_ms + r.enum_ms for r in res)
        lat += [r.prep_ms + r.enum_ms for r in res]
        enum_ms += sum(r.enum_ms for r in res)
        alg += sum(scaled_bytes(r, w.cap) for r in res)
        internal += sum(r.count_internal for r in res)
        h2d += sum(r.h2d_bytes for r in res)
        d2h += sum(r.d2h_bytes for r in res)
        counts = [r.count for r in res]
        bad = [r.status for r in res if r.status not in (0,)]
        if bad:
            raise SystemExit(f"query failures: {bad[:5]}")
    barrier()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    from psm_benchmark_b200.replicas import max_over_ranks
    dev_ms, wall = max_over_ranks([dev_ms, wall], dist, device=f"cuda:{local}")
    nq = len(w.queries)
    value = world * nq * args.steps / (dev_ms / 1e3)
    e2e = world * nq * args.steps / wall
    hbm, peak_kind = peaks()
    achieved = alg / (enum_ms / 1e3) / 1e9 if enum_ms > 0 else 0.0
    line = {"metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic", "config": workload_config(w, world),
            "embeddings_per_s": world * sum(counts) * args.steps / (dev_ms / 1e3),
            # per-query device latency of the plain path (preparation + enumeration)
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(max(lat))},
            "e2e": {"value": e2e, "unit": "queries/s", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps},
            # per plain-path query: prep, enum-init, enum, gather kernels
            "gpu_launches": 4 * nq * args.steps,
            "roofline": {"bound": "hbm", "kernel": "enum_kernel", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_kind": peak_kind,
                         # ncu DRAM bytes per launch (profiles/) against the
                         # algorithmic bytes per launch of this run
                         "traffic": enum_traffic(), "alg_bytes_per_launch": alg / (nq * args.steps),
                         "numerator": "reference-equivalent intersection bytes, scaled to the cap on queries "
                                      "counted past it (bytes x cap / unclamped count)",
                         "counted_past_cap": internal / max(1, sum(counts) * args.steps) - 1.0,
                         # what the captures show bounds the kernel: its rows
                         # stay in L1/L2, so DRAM carries a sliver of the
                         # algorithmic bytes and instruction issue sets the time
                         "limiter": "instruction issue and latency on L1/L2-resident rows (ncu: DRAM bytes "
                                    "about 1/2000 of the algorithmic bytes, L1 hit 97.5 %, 20.5 of 32 threads "
                                    "active per instruction; profiles/enum_kernel_q32_plain_rmat_s20.md)"},
            "clocks": clk}
    # Batched path on the same queries: one preparation launch + one
    # enumeration launch for the whole step (device time, CUDA events).
    bt = 0.0
    bres = None
    for s in range(args.steps + 1 if args.batched else 0):
        flush_l2(flush)
        torch.cuda.synchronize()
        bres = api.match_batch(eng, dg, w.queries, w.method, cap=w.cap, time_limit=args.time_limit)
        if s > 0:
            bt += bres[0].prep_ms + bres[0].enum_ms
    if bres is not None:
        if [r.count for r in bres] != counts:
            raise SystemExit("batched counts differ from the plain path")
        bt = max_over_ranks([bt], dist, device=f"cuda:{local}")[0]
        bval = world * nq * args.steps / (bt / 1e3)
        line["batched"] = {"value": bval, "unit": "queries/s", "ms_per_step": bt / args.steps,
                           "speedup_vs_plain": bval / value, "launches_per_step": 4}
    if world == 1 and args.legs:
        eng.close()
        line["batched_mixed"] = batched_mixed(args, local, w.graph, dg, flush)
        dg.close()
        line["serve"] = serve_run(args, local)
    if world == 1 and args.cpu_baseline and ref_available():
        # the host-core baseline runs once, at N = 1 (rank 0 alone)
        line["cpu_baseline"] = cpu_baseline(w, counts, min(args.cpu_queries, nq))
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


# ------------------------------------------------------ other workloads --
#
# The batched path on 2,000 mixed queries, the serving loop at offered loads
# of 50 / 80 / 95 % of its saturation rate (both also keys of the default
# line at N=1), and the decomposition + join path against the reference's own
# join path (`--workload join`, its own line).

def _torch_setup(local):
    import torch
    torch.cuda.set_device(local)
    return torch


def batched_mixed(args, local, graph=None, dg=None, flush=None):
    """2,000 queries of 4-32 vertices (uniform over {4,6,8,12,16,24,32}) on
    the scale-20 graph: the batched path (one preparation and one
    enumeration launch for all) against the plain path, counts equal."""
    torch = _torch_setup(local)
    from psm_benchmark_b200 import api, gen
    w = gen.batched(num_queries=args.mixed_queries, scale=args.scale, graph=graph)
    # candidate buffers of 2,000 queries take about 40 GB
    eng = api.Engine(device=local, arena_bytes=max(args.arena_gb, 64) << 30)
    own = dg is None
    dg = dg or api.DataGraph.from_graph(w.graph)
    flush = flush if flush is not None else torch.empty(256 << 20 >> 2, dtype=torch.float32, device=f"cuda:{local}")
    nq = len(w.queries)

    def batched():
        flush_l2(flush)
        torch.cuda.synchronize()
        t = time.perf_counter()
        res = api.match_batch(eng, dg, w.queries, w.method, cap=w.cap, time_limit=args.time_limit)
        return res, time.perf_counter() - t

    steps = args.mixed_steps
    # the autotuner picks the batch settings on a sample of the workload
    tune = None
    if args.autotune:
        tune = eng.autotune_batch(dg, w.queries[: args.tune_queries], w.method, cap=w.cap,
                                  time_limit=args.time_limit, repeats=1)
    batched()
    clocks = ClockSampler(local).start()
    dev, wall, res = 0.0, 0.0, None
    for _ in range(steps):
        res, t = batched()
        dev += res[0].prep_ms + res[0].enum_ms
        wall += t
    # the plain path on the same queries (a warm pass over 50, one timed pass)
    for q in w.queries[:50]:
        api.match(eng, dg, q, w.method, cap=w.cap, time_limit=args.time_limit)
    flush_l2(flush)
    torch.cuda.synchronize()
    t = time.perf_counter()
    plain = [api.match(eng, dg, q, w.method, cap=w.cap, time_limit=args.time_limit) for q in w.queries]
    p_wall = time.perf_counter() - t
    clk = clocks.stop()
    p_dev = sum(r.prep_ms + r.enum_ms for r in plain)
    p_enum = sum(r.enum_ms for r in plain)
    if [r.count for r in plain] != [r.count for r in res]:
        raise SystemExit("batched counts differ from the plain path")
    eng.close()
    if own:
        dg.close()
    value = nq * steps / (dev / 1e3)
    sizes = {}
    for q, r in zip(w.queries, plain):
        sizes.setdefault(q.num_vertices, []).append(r.prep_ms + r.enum_ms)
    capped = sum(1 for r in plain if w.cap and r.count >= w.cap)
    return {"metric": "queries/sec (batched GPU path, mixed 4-32-vertex queries, CFL_CFL_EXPLORE, cap 1e9)",
            "value": value, "unit": "queries/s", "steps": steps, "ms_per_step": dev / steps,
            "config": {"workload": "batched_rmat_s20", "queries_per_step": nq,
                       "query_sizes": "uniform over {4,6,8,12,16,24,32}", "method": w.method, "cap": w.cap,
                       "l2": "flushed (256 MiB write) before every step"},
            "embeddings_per_s": sum(r.count for r in res) * steps / (dev / 1e3),
            "e2e": {"value": nq * steps / wall, "unit": "queries/s"},
            "gpu_launches_per_step": 4,
            "plain": {"value": nq / (p_dev / 1e3), "e2e": nq / p_wall, "unit": "queries/s",
                      "latency_ms_by_size": {str(k): {"p50": float(np.percentile(v, 50)),
                                                      "p99": float(np.percentile(v, 99))}
                                             for k, v in sorted(sizes.items())}},
            "speedup_vs_plain": value / (nq / (p_dev / 1e3)),
            "e2e_speedup_vs_plain": (nq * steps / wall) / (nq / p_wall),
            # batching removes per-query preparation launches and overlaps
            # enumeration tails; the enumeration work itself remains: the
            # plain path's device time over its enumeration time is the
            # speed-up from removing the preparation cost alone
            "plain_enum_share": p_enum / p_dev, "plain_device_over_enum": p_dev / p_enum,
            "counts_equal_plain": True, "capped_queries": capped, "clocks": clk,
            "autotune": ({"sample_queries": min(nq, args.tune_queries), "best": tune["best"], "tried": tune["tried"]}
                         if tune else None)}


def batched_leg(args, local):
    line = batched_mixed(args, local)
    line.update({"n_gpus": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "dtype": "u32", "data": "synthetic", "gpu_launches": 4 * line["steps"]})
    print(json.dumps(line))


def join_leg(args, local):
    _torch_setup(local)
    from psm_benchmark_b200 import api, gen
    from psm_benchmark_b200.graphs import Graph
    golden = ROOT / "tests" / "golden"
    ref = json.loads((golden / "join_ref.json").read_text())
    z = np.load(golden / "hprd15.npz")
    hg = Graph(off=z["off"], nbr=z["nbr"], labels=z["labels"])
    hq = []
    for lab, e in zip(z["q_labels"], z["q_edges"]):
        e = e[e[:, 0] >= 0]
        hq.append(Graph.from_edges(len(lab), lab, e))
    rg = gen.make_graph("rmat", 2, scale=12, edge_factor=8, num_labels=32)
    rq = [(Graph.from_edges(len(e["query"]["labels"]), e["query"]["labels"], e["query"]["edges"]), e["count"])
          for e in ref["rmat12"]["queries"] if e["count"] is not None]
    eng = api.Engine(device=local, arena_bytes=args.arena_gb << 30)
    cases = [(api.DataGraph.from_graph(hg), q, c, 4) for q, c in zip(hq, ref["hprd"])]
    rdg = api.DataGraph.from_graph(rg)
    cases += [(rdg, q, c, 12) for q, c in rq]
    for _ in range(args.warmup):
        for dg, q, c, mu in cases:
            api.match_join(eng, dg, q, "CFL_CFL_EXPLORE", max_unit_vertices=mu)
    dev, wall = 0.0, 0.0
    for _ in range(args.steps):
        for dg, q, c, mu in cases:
            t = time.perf_counter()
            r = api.match_join(eng, dg, q, "CFL_CFL_EXPLORE", max_unit_vertices=mu)
            wall += time.perf_counter() - t
            dev += r.prep_ms + r.enum_ms + r.join_ms
            if r.count != c:
                raise SystemExit(f"join count {r.count} differs from the reference's {c}")
    n = len(cases) * args.steps
    line = {"metric": "queries/sec (decomposition + hash-join path)", "value": n / (dev / 1e3), "unit": "queries/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": "join_hprd_rmat12",
                       "queries": f"{len(hq)} HPRD-15 (units <= 4 vertices) + {len(rq)} R-MAT scale-12 queries of "
                                  "16-24 vertices (units <= 12) that the reference's join path finishes",
                       "method": "CFL_CFL_EXPLORE", "counts": "equal to the reference's -QorCandi Q counts"},
            "e2e": {"value": n / wall, "unit": "queries/s"}}
    if args.cpu_baseline and ref_available():
        tmp = Path(tempfile.mkdtemp(prefix="psmjoin_"))
        d = tmp / "a" / "b" / "c"
        (d / "q").mkdir(parents=True)
        files = {}
        tot, nref = 0.0, 0
        for k, (dg, q, c, mu) in enumerate(cases):
            g = hg if k < len(hq) else rg
            key = "h" if k < len(hq) else "r"
            if key not in files:
                files[key] = d / f"{key}.txt"
                gen.write_text(g, files[key])
            qp = d / "q" / f"q{k}.txt"
            q.write_text(qp)
            log = tmp / "log.txt"
            if log.exists():
                log.unlink()
            subprocess.run([str(REF_BIN), "-d", str(files[key]), "-q", str(qp), "-num", "MAX", "-time_limit", "120",
                            "-OutputFile", str(log), "-QorCandi", "Q", "-Qpattern", "STAR", "-JoinMethod", "LEFTDEEP",
                            "-threadnums", "1", "-BackMethods", "CFL_CFL_EXPLORE"], check=True, capture_output=True,
                           timeout=300)
            text = log.read_text()
            tot += float(re.findall(r"Total time \(seconds\): ([0-9.e+-]+)", text)[-1])
            nref += 1
            if tot > 60:
                break
        line["cpu_baseline"] = {"value": nref / tot, "unit": "queries/s", "cores": 1, "kind": "reference",
                                "sample": f"{nref} queries through the reference's join path (-QorCandi Q -Qpattern "
                                          f"STAR -JoinMethod LEFTDEEP -threadnums 1), {tot:.2f} s Total time"}
    print(json.dumps(line))


def join4_leg(args, local):
    """Config-4-shaped decomposition + join: R-MAT (edge factor 16, 64
    Zipf(1.0) labels) at a reduced scale, 24-32-vertex random-walk queries,
    the cost-based bounded decomposition (units <= 12 vertices) joined bushy,
    each query under a time limit; counts checked against the plain path on
    the same queries and, on a bounded sample, the reference's own join path
    (-QorCandi Q)."""
    _torch_setup(local)
    from psm_benchmark_b200 import api, gen
    w = gen.join(num_queries=args.join_queries, scale=args.join_scale)
    eng = api.Engine(device=local, arena_bytes=max(args.arena_gb, 64) << 30)
    dg = api.DataGraph.from_graph(w.graph)
    rows = []
    for i, q in enumerate(w.queries):
        t = time.perf_counter()
        try:
            r = api.match_join(eng, dg, q, w.method, max_unit_vertices=12, pattern="COST", join_method="BUSHY",
                               time_limit=args.join_limit)
            jt = time.perf_counter() - t
            jres = (r.count, r.prep_ms + r.enum_ms + r.join_ms, jt, len(r.units))
        except Exception as e:  # time limit or arena: the query did not finish
            jres = (None, None, time.perf_counter() - t, str(e)[:60])
        p = api.match(eng, dg, q, w.method, cap=0, time_limit=args.join_limit)
        rows.append({"i": i, "n": q.num_vertices, "join": jres, "plain": (None if p.overtime else p.count,
                                                                         p.prep_ms + p.enum_ms)})
    done = [r for r in rows if r["join"][0] is not None]
    agree = sum(1 for r in done if r["plain"][0] is not None and r["plain"][0] == r["join"][0])
    both = sum(1 for r in done if r["plain"][0] is not None)
    if agree != both:
        raise SystemExit("join counts differ from the plain path")
    dev_s = sum(r["join"][1] for r in done) / 1e3
    line = {"metric": "queries/sec (decomposition + hash-join path, config-4 shape)",
            "value": len(done) / dev_s if dev_s else 0.0, "unit": "queries/s", "n_gpus": 1, "steps": 1,
            "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": "join_rmat", "graph": f"R-MAT scale {args.join_scale}, edge factor 16, "
                                                         "64 Zipf(1.0) labels",
                       "edges": w.graph.num_edges, "queries": len(w.queries), "query_sizes": "24-32",
                       "pattern": "COST (units <= 12), BUSHY", "time_limit_s": args.join_limit},
            "finished": len(done), "counts_checked_vs_plain": both,
            "plain_finished": sum(1 for r in rows if r["plain"][0] is not None),
            "per_query": rows}
    if args.cpu_baseline and ref_available():
        tmp = Path(tempfile.mkdtemp(prefix="psmjoin4_"))
        d = tmp / "a" / "b" / "c"
        (d / "q").mkdir(parents=True)
        gen.write_text(w.graph, d / "g.txt")
        ref = []
        for r in rows[: args.join_ref_queries]:
            qp = d / "q" / f"q{r['i']}.txt"
            w.queries[r["i"]].write_text(qp)
            log = tmp / "log.txt"
            if log.exists():
                log.unlink()
            subprocess.run([str(REF_BIN), "-d", str(d / "g.txt"), "-q", str(qp), "-num", "MAX", "-time_limit",
                            str(int(args.join_limit)), "-OutputFile", str(log), "-QorCandi", "Q", "-Qpattern", "STAR",
                            "-JoinMethod", "LEFTDEEP", "-threadnums", "1", "-BackMethods", w.method],
                           capture_output=True, timeout=args.join_limit + 300)
            text = log.read_text() if log.exists() else ""
            c = re.findall(r"#Embeddings: (\d+)", text)
            o = re.findall(r"Overtime: (\d+)", text)
            t = re.findall(r"Total time \(seconds\): ([0-9.e+-]+)", text)
            fin = bool(c and o and o[-1] == "0")
            ref.append({"i": r["i"], "count": int(c[-1]) if fin else None, "total_s": float(t[-1]) if t else None})
            if fin and r["join"][0] is not None and int(c[-1]) != r["join"][0]:
                raise SystemExit(f"join count differs from the reference's (query {r['i']})")
        line["reference"] = {"runs": ref, "finished": sum(1 for x in ref if x["count"] is not None),
                             "note": "-QorCandi Q -Qpattern STAR -JoinMethod LEFTDEEP -threadnums 1"}
    eng.close()
    dg.close()
    print(json.dumps(line))


def serve_run(args, local):
    """Serving on R-MAT scale 24 (edge factor 16, 128 uniform labels): the
    request stream all at once (saturation), then as Poisson arrivals at 50,
    80 and 95 % of that rate; latency = completion - scheduled arrival."""
    _torch_setup(local)
    from psm_benchmark_b200 import api, gen
    nq = args.serve_queries
    scale = args.serve_scale
    t = time.time()
    w = gen.serve(num_queries=nq, scale=scale)
    dg = api.DataGraph.from_graph(w.graph)
    setup_s = time.time() - t
    lanes = args.lanes
    srv = api.Server(dg, w.method, cap=w.cap, time_limit=args.time_limit, lanes=lanes, max_batch=args.max_batch,
                     lane_arena_bytes=(args.serve_budget_gb << 30) // lanes, full_gpu_lanes=not args.serve_share)
    clocks = ClockSampler(local).start()
    # warm-up, then saturation: everything queued at once
    for q in w.queries[: min(nq, 500)]:
        srv.submit(q)
    srv.drain(min(nq, 500))
    t0 = api.Server.clock_ns()
    for q in w.queries:
        srv.submit(q)
    res = srv.drain(nq, timeout_s=3600)
    if len(res) != nq:
        raise SystemExit(f"serving: {len(res)} of {nq} results")
    sat_span = (max(r.done_ns for r in res) - t0) / 1e9
    sat = nq / sat_span
    base = min(r.ticket for r in res)
    counts = {r.ticket - base: r.count for r in res}
    sat_lat = [(r.done_ns - t0) / 1e6 for r in res]
    # batches of the saturation run: (lane, start) -> size, wall span until
    # the batch's last result
    batches = {}
    for r in res:
        k = (r.lane, r.start_ns)
        size, end = batches.get(k, (r.batch_size, 0))
        batches[k] = (size, max(end, r.done_ns))
    lane_busy = {}
    for (ln, st), (_, end) in batches.items():
        lane_busy[ln] = lane_busy.get(ln, 0.0) + (end - st) / 1e9
    spans = [(end - st) / 1e6 for (_, st), (_, end) in batches.items()]
    # idle time of a lane between its batches (last result to next start)
    gaps = []
    for ln in set(k[0] for k in batches):
        seq = sorted((st, end) for (l2, st), (_, end) in batches.items() if l2 == ln)
        gaps += [(b[0] - a[1]) / 1e6 for a, b in zip(seq, seq[1:])]
    batch_stats = {"batches": len(batches), "mean_batch": float(np.mean([b[0] for b in batches.values()])),
                   "span_ms": {"p50": float(np.percentile(spans, 50)), "p99": float(np.percentile(spans, 99)),
                               "max": float(max(spans))},
                   "lane_busy_frac": {str(k): v / sat_span for k, v in sorted(lane_busy.items())},
                   "lane_gap_ms": {"p50": float(np.percentile(gaps, 50)) if gaps else 0.0,
                                   "max": float(max(gaps)) if gaps else 0.0}}
    loads = {}
    for load in args.serve_loads:
        rate = load * sat
        arrive = gen.poisson_arrivals(nq, rate, w.seed + int(load * 100))
        start = api.Server.clock_ns()
        sched = {}
        for i, (q, a) in enumerate(zip(w.queries, arrive)):
            target = start + int(a * 1e9)
            while api.Server.clock_ns() < target:
                time.sleep(min(0.0005, max(0.0, (target - api.Server.clock_ns()) / 1e9)))
            tk = srv.submit(q)
            sched[tk] = (i, target)
        out = srv.drain(nq, timeout_s=3600)
        if len(out) != nq:
            raise SystemExit(f"serving at {load}: {len(out)} of {nq} results")
        lat = [(r.done_ns - sched[r.ticket][1]) / 1e6 for r in out]
        bad = sum(1 for r in out if r.count != counts[sched[r.ticket][0]])
        if bad:
            raise SystemExit(f"serving at {load}: {bad} counts differ from the saturation run")
        span = (max(r.done_ns for r in out) - start) / 1e9
        sizes = {}
        for r, l in zip(out, lat):
            sizes.setdefault(w.queries[sched[r.ticket][0]].num_vertices, []).append(l)
        loads[f"{int(round(load * 100))}%"] = {
            "offered_qps": rate, "achieved_qps": nq / span, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(max(lat)),
            "p99_ms_by_size": {str(k): float(np.percentile(v, 99)) for k, v in sorted(sizes.items())},
            "mean_batch": float(np.mean([r.batch_size for r in out])), "counts_equal_saturation_run": True}
    clk = clocks.stop()
    srv.close()
    # the plain path (one query per launch sequence, whole GPU) on the first
    # requests of the same stream, for the served / plain ratio
    plain = None
    if args.serve_plain > 0:
        eng = api.Engine(device=local, arena_bytes=args.arena_gb << 30)
        sample = w.queries[: min(nq, args.serve_plain)]
        for q in sample[:20]:
            api.match(eng, dg, q, w.method, cap=w.cap, time_limit=args.time_limit)
        t = time.perf_counter()
        pres = [api.match(eng, dg, q, w.method, cap=w.cap, time_limit=args.time_limit) for q in sample]
        p_wall = time.perf_counter() - t
        eng.close()
        p_dev = sum(r.prep_ms + r.enum_ms for r in pres) / 1e3
        bad = sum(1 for i, r in enumerate(pres) if r.count != counts[i])
        if bad:
            raise SystemExit(f"serving: {bad} counts differ from the plain path")
        plat = [r.prep_ms + r.enum_ms for r in pres]
        plain = {"queries": len(sample), "value": len(sample) / p_dev, "e2e": len(sample) / p_wall,
                 "latency_ms": {"p50": float(np.percentile(plat, 50)), "p99": float(np.percentile(plat, 99)),
                                "max": float(max(plat))},
                 "unit": "queries/s", "served_saturation_vs_plain_e2e": sat / (len(sample) / p_wall),
                 "counts_equal_served": True}
    dg.close()
    return {"metric": "queries/sec and p50/p99 latency (serving, continuous batching)", "value": sat,
            "unit": "queries/s",
            "config": {"workload": "serve_rmat", "graph": f"R-MAT scale {scale}, edge factor 16, 128 uniform labels",
                       "edges": w.graph.num_edges, "queries": nq,
                       "query_sizes": "{4,8,12,16,24,32} weighted .3/.25/.2/.1/.1/.05", "cap": w.cap,
                       "lanes": lanes, "max_batch": args.max_batch, "budget_gb": args.serve_budget_gb,
                       "lane_grid": "1/lanes of the GPU" if args.serve_share else "whole GPU",
                       "setup_s": setup_s},
            "saturation_qps": sat, "saturation_span_s": sat_span,
            "saturation_latency_ms": {"p50": float(np.percentile(sat_lat, 50)),
                                      "p99": float(np.percentile(sat_lat, 99))},
            "saturation_batches": batch_stats,
            "loads": loads, "plain": plain, "clocks": clk}


def serve_leg(args, local):
    line = serve_run(args, local)
    line.update({"n_gpus": 1, "steps": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak",
                 "vs_baseline": None, "dtype": "u32", "data": "synthetic"})
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--queries", type=int, default=200)
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--time-limit", type=float, default=600.0)
    ap.add_argument("--arena-gb", type=int, default=8)
    ap.add_argument("--ref-limit", type=int, default=600, help="reference time limit per query (s)")
    ap.add_argument("--ref-mt-limit", type=int, default=10,
                    help="time limit of the one multi-threaded reference run (s); 0 = skip")
    ap.add_argument("--cpu-queries", type=int, default=16, help="whole queries in the cpu_baseline sample")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-batched", dest="batched", action="store_false")
    ap.add_argument("--no-legs", dest="legs", action="store_false",
                    help="leave out the batched_mixed and serve keys of the default line")
    ap.add_argument("--only", default="", help="comma-separated query indices (profiling runs)")
    ap.add_argument("--intersect", default="BINARY", choices=["BINARY", "AUTO", "MERGE"],
                    help="intersection variant of the plain path's enumeration kernel")
    ap.add_argument("--workload", default="plain", choices=["plain", "batched", "join", "join4", "serve"])
    ap.add_argument("--join-scale", type=int, default=11)
    ap.add_argument("--join-queries", type=int, default=12)
    ap.add_argument("--join-limit", type=float, default=5.0)
    ap.add_argument("--join-ref-queries", type=int, default=6)
    ap.add_argument("--mixed-queries", type=int, default=2000)
    ap.add_argument("--mixed-steps", type=int, default=2)
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="leave the batched path's settings at their defaults")
    ap.add_argument("--tune-queries", type=int, default=300, help="sample of the mixed workload for the autotuner")
    ap.add_argument("--serve-queries", type=int, default=50000)
    ap.add_argument("--serve-scale", type=int, default=24)
    ap.add_argument("--serve-plain", type=int, default=2000,
                    help="requests of the stream also run through the plain path (served / plain ratio)")
    ap.add_argument("--serve-loads", type=lambda s: [float(x) for x in s.split(",")], default=[0.5, 0.8, 0.95])
    ap.add_argument("--lanes", type=int, default=4, help="serving lanes")
    ap.add_argument("--max-batch", type=int, default=64, help="serving batch limit")
    ap.add_argument("--serve-budget-gb", type=int, default=120, help="serving device-memory budget")
    ap.add_argument("--serve-share", action="store_true",
                    help="size each serving lane's grids to 1/lanes of the GPU (else every lane launches whole-GPU grids)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.workload != "plain":
        if args.impl == "reference" or world > 1:
            if rank == 0:
                print(json.dumps({"impl": args.impl, "unavailable": "the batched, join and serve workloads run on "
                                                                     "one GPU through this arm only"}))
            return
        {"batched": batched_leg, "join": join_leg, "join4": join4_leg,
         "serve": serve_leg}[args.workload](args, dist_setup()[2])
        return
    if args.impl == "reference":
        reference_arm(args, world, rank)
    else:
        ours_arm(args, world, rank, local)


if __name__ == "__main__":
    main()
