#!/usr/bin/env python3
"""Benchmark of the delta-stepping SSSP path on B200.

Default run (N=1, ``--workload all``): ONE JSON line whose headline
``value`` is the plain single-source solve on the planar road-like kNN graph
(6.3M points uniform in the unit square, 3 nearest neighbours symmetrised,
w = round(1e6*d)+1, 5 seeded sources solved one at a time, configuration
tuned on other sources) and which carries three more measured blocks:

  "c3"       plain solves on R-MAT scale 22 (edge factor 16, w U{1..2^20}),
  "batched"  64 sources on a 4896^2 road-like grid in one persistent launch
             replayed from a CUDA graph, against 64 back-to-back plain solves,
  "served"   continuous batching over 8 HBM-resident graphs under Poisson
             arrivals (100/s and 1000/s offered, and a saturating burst),
             p50/p99 latency, against back-to-back plain solves of the mix.

Every result of every block is checked against the CPU oracle outside the
timed regions: plain and batched distances element by element, served
results by the device-computed digest of each distance array against the
digest of the oracle's distances (``correct``).  Each block has its own
clock record, sampled while its timed work ran.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mlmq|reference]
                  [--workload all|c1|c2|c3|c4|c5] [--skip c3,batched,served]

* value: GTEPS = arcs out of reached vertices (the oracle's total_work) /
  summed device time of the solves, CUDA events on the launch stream, inputs
  resident in HBM, L2 flushed (256 MiB write) between solves.
* e2e: the same metric through mlmq_solve_host() with pinned host buffers:
  CSR upload, every solve, every distance copy back.
* roofline: algorithmic bytes per solve 12*m_r + 12*n_r over the kernel's
  average duration, against the measured HBM copy bandwidth.
* cpu_baseline: the reference's own sssp_sequential (oracle/_ref) -- or the
  oracle port when it was not built -- on the host, one thread.
* --impl reference: the reference's CPU implementation alone, one host
  thread per source, on the headline workload and metric.

Multi-GPU (torchrun): replicas only -- every rank solves the same headline
job on its own GPU with no collective on the data path; time is the max over
ranks.  The c3/batched/served blocks are measured at N=1 only.
"""
import argparse
import csv
import io
import json
import os
import platform
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SSSP GTEPS (plain single-source delta-stepping, queries one at a time)"
BATCH_METRIC = "SSSP queries/sec (batched: 64 sources in one persistent launch)"
SERVE_METRIC = "SSSP queries/sec (served: continuous batching over 8 HBM-resident graphs)"
WORKLOAD_TEXT = {
    "c1": "grid 512x512, 4-neighbour, 10% undirected edges dropped, w U{1000..100000}, "
          "source 0, delta 200000, L1SLF_L2DQ",
    "c2": "kNN road-like: 6.3M points U[0,1)^2, k=3 symmetrised, w=round(1e6*d)+1, "
          "5 seeded sources one at a time, delta autotuned around 200000, L1SLF_L2DQ",
    "c3": "R-MAT scale 22, edge factor 16, (.57,.19,.19,.05), dedup, no self-loops, "
          "w U{1..2^20}, 5 seeded sources one at a time, delta autotuned, L1SLF_L2DQ",
    "c4": "batched: 64 seeded sources on a 4896x4896 grid (10% edges dropped, "
          "w U{1000..100000}) in one persistent launch replayed from a CUDA graph, "
          "64 int32 distance arrays, vs 64 back-to-back plain solves",
    "c5": "served: grids 2^16..2^24 + R-MAT 18/20/22 resident; Poisson arrivals, graph and "
          "source uniform per query",
}
# Scaled-down workloads for functional runs of the whole bench (--small).
SMALL = {"c2_points": 200_000, "c3_scale": 16, "c4_side": 1024, "c5_max_log2": 18,
         "c5_rmat": (14, 16)}


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("mlmq", "reference"), default="mlmq")
    ap.add_argument("--workload", choices=("all", "c1", "c2", "c3", "c4", "c5"), default="all")
    ap.add_argument("--skip", default="", help="all: blocks to leave out (c3,batched,served)")
    ap.add_argument("--small", action="store_true",
                    help="scaled-down workloads (functional runs of the whole bench)")
    ap.add_argument("--served-rate", type=float, default=1000.0,
                    help="served: offered arrival rate of the latency run (queries/s)")
    ap.add_argument("--served-queries", type=int, default=1000,
                    help="served: queries in each of the two runs")
    ap.add_argument("--burst-rate", type=float, default=20000.0,
                    help="served: arrival rate of the saturating run (queries/s)")
    ap.add_argument("--light-rate", type=float, default=100.0,
                    help="served: arrival rate of the light-load run (queries/s)")
    ap.add_argument("--light-queries", type=int, default=200,
                    help="served: queries in the light-load run")
    ap.add_argument("--slots", type=int, default=64)
    ap.add_argument("--slot-warps", type=int, default=8, help="served: worker warps per CTA")
    ap.add_argument("--sources", type=int, default=0, help="limit the number of sources")
    ap.add_argument("--side", type=int, default=0,
                    help="c4: grid side instead of 4896 (small cases for profiler captures)")
    ap.add_argument("--scale", type=int, default=0,
                    help="c3: R-MAT scale instead of 22 (small cases for profiler captures)")
    ap.add_argument("--batch-steps", type=int, default=10, help="batched: timed launches")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--config", default="",
                    help="c1-c3: JSON overrides of the solver configuration, used instead of "
                         "tuning (reproducible profiler runs)")
    return ap.parse_args(argv)


# ---- measurement helpers ----------------------------------------------------------

def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kernel, workload, delta=None):
    """Per-launch DRAM bytes from the committed ncu summary, if captured:
    (bytes, delta of the captured configuration or None).  A workload may
    have captures at several bucket widths (`delta=N` after the bytes); the
    one at the tuned delta is taken, else the nearest."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    found = []
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
                    tag = None
                    if len(parts) >= 4 and parts[3].startswith("delta="):
                        tag = int(parts[3][len("delta="):])
                    found.append((float(parts[2]), tag))
    except OSError:
        pass
    if not found:
        return None, None
    if delta is None or all(t is None for _, t in found):
        return found[0]
    tagged = [f for f in found if f[1] is not None]
    return min(tagged, key=lambda f: abs(f[1] - int(delta)))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms while running."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = tempfile.TemporaryFile(mode="w+")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.out.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.out.read())) if len(r) >= 9]
        if not rows:
            return None

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows]
        util = [num(r[4]) for r in rows]
        loaded = [s for s, u in zip(sm, util) if s is not None and (u or 0) > 0] or \
                 [s for s in sm if s is not None]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": float(np.median(loaded)) if loaded else None,
                "sm_max_mhz": num(rows[0][2]), "reasons": reasons, "samples": len(rows)}


def host_cpu():
    """Model name and core count of this host (for CPU figures)."""
    model = platform.processor() or ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def oracle_lib():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    return ol


def cpu_reference_gteps(g, srcs, threads):
    """Times the reference's sssp_sequential (or the oracle port) on the host."""
    ol = oracle_lib()
    fn = ol.ref_sequential if ol.reference() is not None else ol.sssp_i32
    kind = "reference" if ol.reference() is not None else "port"

    def one(src):
        t0 = time.perf_counter()
        _, work = fn(g, src)
        return work, time.perf_counter() - t0

    t0 = time.perf_counter()
    if threads <= 1:
        res = [one(s) for s in srcs]
    else:
        with ThreadPoolExecutor(threads) as ex:
            res = list(ex.map(one, srcs))
    wall = time.perf_counter() - t0
    work = sum(r[0] for r in res)
    busy = sum(r[1] for r in res)
    return work, wall, busy, kind


def graph_digest(g):
    """Fingerprint of a CSR (row, col, w), so both arms can show they ran the
    same graph."""
    import hashlib
    h = hashlib.sha256()
    for a in (g.row, g.col, g.w):
        h.update(np.ascontiguousarray(a, dtype=np.int32).tobytes())
    return h.hexdigest()[:16]


def cfg_summary(cfg, keys=("delta", "warps_per_block", "work_blocks", "relax_unroll",
                           "vertex_tiles", "l1_ahead", "light_heavy", "bucket_sync", "l2_batch",
                           "topup", "queue_type")):
    d = {k: getattr(cfg, k) for k in keys}
    d["queue"] = "L1SLF_L2DQ" if d.pop("queue_type") == 19 else "L1V_L2DQ"
    return d


# ---- workloads -------------------------------------------------------------------

def headline_workload(args):
    """The headline (C2 unless --workload c1/c3) graph and timed sources."""
    from mlmq_tpds_withl3_b200 import workloads
    name = args.workload if args.workload in ("c1", "c2", "c3") else "c2"
    if name == "c1":
        g, srcs = workloads.c1()
    elif name == "c2":
        g, srcs = workloads.c2(points=SMALL["c2_points"]) if args.small else workloads.c2()
    else:
        scale = args.scale or (SMALL["c3_scale"] if args.small else 22)
        g, srcs = workloads.c3(scale=scale)
    if args.sources:
        srcs = srcs[:args.sources]
    return name, g, srcs


def _largest_component(g):
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components
    a = csr_matrix((np.ones(g.m, np.int8), g.col, g.row), shape=(g.n, g.n))
    _, labels = connected_components(a, directed=True, connection="weak")
    return np.flatnonzero(labels == np.bincount(labels).argmax())


def _seeded(pool, count, seed=1):
    rng = np.random.default_rng(seed)
    if count >= len(pool):
        return [int(v) for v in pool[:count]]
    return [int(v) for v in rng.choice(pool, size=count, replace=False)]


def reference_workload(args):
    """The headline graph and sources for the reference arm, built by the
    oracle's C restatement of the generators (oracle/workload.c) so that the
    reference arm never loads the product library; the source rule is the
    one mlmq_tpds_withl3_b200.workloads applies (tests/test_bench_host.py
    checks that both arms get the same graph and sources)."""
    ol = oracle_lib()
    name = args.workload if args.workload in ("c1", "c2", "c3") else "c2"
    if name == "c1":
        g, srcs = ol.gen_grid(512, 512, 0.10, 1000, 100000, 1), [0]
    elif name == "c2":
        g = ol.gen_knn(SMALL["c2_points"] if args.small else 6_300_000, 3, 1e6, 1)
        srcs = _seeded(_largest_component(g), 5)
    else:
        g = ol.gen_rmat(args.scale or (SMALL["c3_scale"] if args.small else 22), 16, 0.57, 0.19,
                        0.19, 1, 1 << 20, 1)
        comp = _largest_component(g)
        srcs = _seeded(comp[np.diff(g.row)[comp] > 0], 5)
    if args.sources:
        srcs = srcs[:args.sources]
    return name, g, srcs


def workload_config(name, g, srcs, small):
    """The workload keys of `config`, identical in both arms."""
    text = WORKLOAD_TEXT[name] + (" [scaled down: --small]" if small else "")
    if name == "c3" and g.n != 1 << 22 and not small:
        text = text.replace("scale 22", f"scale {g.n.bit_length() - 1} [scaled down: --scale]")
    return {"workload": text, "n": g.n, "m": g.m, "sources": [int(s) for s in srcs],
            "graph_sha256_16": graph_digest(g)}


# ---- plain single-source arm -------------------------------------------------------

def plain_arm(args, name, g, srcs, rep, local, steps, warmup, cpu_baseline, e2e_on):
    """Tuned plain solves of `srcs` on `g`, one at a time.  Returns a dict of
    JSON fields (value in GTEPS, roofline, e2e, correct, clocks ...)."""
    import torch
    from mlmq_tpds_withl3_b200 import DeviceGraph, Solver, autotune, default_config, workloads
    from mlmq_tpds_withl3_b200._lib import check, lib
    from mlmq_tpds_withl3_b200.replicas import whole_job_rate
    ol = oracle_lib()
    world = rep.world

    dg = DeviceGraph.upload(g)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flush_l2():
        flush.zero_()
        torch.cuda.synchronize()

    tune_report = None
    if args.config:
        cfg = default_config(**{"delta": 200000, **json.loads(args.config)})
    elif name == "c1" or args.no_tune:
        cfg = default_config(delta=200000)
    else:
        # Rank 0 tunes; every replica then runs its configuration.
        if rep.rank == 0:
            pool = workloads.c3_source_pool(g) if name == "c3" else None
            probes = workloads.probe_sources(g, srcs, count=4, pool=pool)
            cfg, tune_report = autotune.tune(dg, g, probes, kind=name, use_cache=False,
                                             between=flush_l2)
        picked = rep.broadcast(cfg.as_dict() if rep.rank == 0 else None)
        cfg = default_config(**picked)
        # Tuning leaves the pool holding blocks of every candidate's sizes.
        lib.mlmq_release_cached()
    solver = Solver(dg, cfg)

    # Correctness and per-query work (oracle, untimed): every timed source.
    dists, works = ol.sssp_many(g, srcs, threads=min(len(srcs), os.cpu_count() or 1))
    reached = (dists != ol.INT_MAX).sum(axis=1)
    correct = True
    for k, s in enumerate(srcs):
        solver.solve(s)
        if not np.array_equal(solver.dist(), dists[k]):
            correct = False

    stream = torch.cuda.Stream()

    def step(events):
        for s in srcs:
            with torch.cuda.stream(stream):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solver.launch(s, stream.cuda_stream)
            e1.record(stream)
            solver.wait()
            if events is not None:
                events.append((e0, e1))

    for _ in range(warmup):
        step(None)
    torch.cuda.synchronize()
    rep.barrier()
    events = []
    sampler = ClockSampler(local)
    with sampler:
        t_wall0 = time.perf_counter()
        for _ in range(steps):
            step(events)
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall0
    rep.barrier()
    per_query_ms = np.array([a.elapsed_time(b) for a, b in events])
    total_s = rep.max(per_query_ms.sum() / 1e3)
    work_step = float(np.sum(works))
    gteps = whole_job_rate(work_step * steps, world, total_s) / 1e9

    # Roofline of the persistent kernel.
    bytes_q = 12.0 * np.asarray(works, np.float64) + 12.0 * reached.astype(np.float64)
    launch_s = per_query_ms / 1e3
    achieved_gbs = float(np.sum(np.tile(bytes_q, steps)) / np.sum(launch_s) / 1e9)
    peak, peak_kind = measured_peak()
    traffic, traffic_delta = ncu_traffic("sssp_plain_kernel", name, cfg.delta)
    stats = solver.stats()
    solver.close()

    # End to end through the host-buffer API (the pool starts from what the
    # call itself needs; warm-up calls grow it).
    e2e = None
    if e2e_on:
        lib.mlmq_release_cached()
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        row, col, w = pin(g.row), pin(g.col), pin(g.w)
        src_arr = np.asarray(srcs, np.int32)
        out = torch.empty((len(srcs), g.n), dtype=torch.int32).pin_memory()
        e2e_steps = max(3, min(steps, 9))
        # Warm-up calls as for the device timing: the first calls after tuning
        # grow the library's memory pool to the call's working set and load
        # the upload's sort kernels (R-MAT-22: the first calls took 90-650 ms
        # against ~44 ms later; the PCIe copy, shared with the host's other
        # GPUs, varies from call to call too).
        e2e_warm = max(3, min(warmup, 5))
        walls = []
        for i in range(e2e_steps + e2e_warm):
            t0 = time.perf_counter()
            check(lib.mlmq_solve_host(g.n, g.m, row.data_ptr(), col.data_ptr(), w.data_ptr(),
                                      len(srcs), src_arr.ctypes.data, out.data_ptr(), cfg),
                  "mlmq_solve_host")
            if i >= e2e_warm:
                walls.append(time.perf_counter() - t0)
        # The median step: the PCIe link and the host are shared with the
        # machine's other GPUs and their jobs, and single calls now and then
        # take 2-10x longer for it (every wall is listed, with the mean).
        e2e_s = rep.max(float(np.median(walls)))
        e2e_mean = rep.max(float(np.mean(walls)))
        correct = correct and np.array_equal(out.numpy(), dists)
        e2e = {"value": whole_job_rate(work_step, world, e2e_s) / 1e9,
               "unit": "GTEPS",
               "h2d_bytes_per_step": int(4 * (g.n + 1) + 8 * g.m),
               "d2h_bytes_per_step": int(4 * g.n * len(srcs)),
               "ms_per_step": e2e_s * 1e3,
               "statistic": "median of the steps",
               "mean_ms_per_step": e2e_mean * 1e3,
               "value_from_mean": whole_job_rate(work_step, world, e2e_mean) / 1e9,
               "walls_ms": [round(x * 1e3, 2) for x in walls],
               "warmup_calls": e2e_warm,
               "api": "mlmq_solve_host (pinned host CSR in, distances out)"}
        del out, row, col, w
    del dists
    dg.close()

    cpu = None
    if cpu_baseline and rep.rank == 0 and world == 1:
        work, wall, _, kind = cpu_reference_gteps(g, srcs, 1)
        cpu = {"value": work / wall / 1e9, "unit": "GTEPS", "cores": 1, "kind": kind,
               "host_cpu": host_cpu(),
               "sample": f"{len(srcs)} sources of the same workload, one after another, "
                         f"{wall:.1f} s"}

    out = {
        "value": gteps, "unit": "GTEPS", "steps": steps, "warmup": warmup,
        "ms_per_step": total_s / steps * 1e3,
        "config": workload_config(name, g, srcs, args.small),
        "solver": {**cfg_summary(cfg), "grid": stats["grid"], "block": stats["block"],
                   "l2_between_solves": "flushed (256 MiB write, outside the timed events)"},
        "correct": bool(correct),
        "checked": f"every timed source ({len(srcs)}) element by element against the oracle, "
                   f"device-resident and through mlmq_solve_host",
        "qps": whole_job_rate(len(srcs) * steps, world, total_s),
        "latency_ms": {"p50": float(np.percentile(per_query_ms, 50)),
                       "p99": float(np.percentile(per_query_ms, 99))},
        "work_per_step": int(work_step),
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak, "traffic": traffic,
                     "traffic_capture": (f"one ncu capture at delta {traffic_delta}"
                                         if traffic_delta is not None else "one ncu capture"),
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "kernel": "sssp_plain_kernel",
                     "algorithmic_bytes_per_launch": float(np.mean(bytes_q))},
        "e2e": e2e, "cpu_baseline": cpu, "clocks": sampler.summary(),
        "gpu_launches": len(events), "wall_s_timed_region": t_wall,
        "relax_per_arc": float(stats["relaxed"]) / max(1.0, float(works[-1])),
        "last_solve_stats": {k: int(stats[k]) for k in ("relaxed", "improved", "pushed",
                                                         "l3_pushed", "batches", "idle")},
    }
    if tune_report:
        trials = sorted(tune_report.get("trials", []), key=lambda t: t["seconds"])
        out["autotune"] = {"config": tune_report.get("config"),
                           "probe_sources": tune_report.get("probe"),
                           "trials": len(trials),
                           "fastest": [{"config": t["config"], "ms": round(t["seconds"] * 1e3, 2)}
                                       for t in trials[:4]]}
    return out


# ---- batched arm (C4) ----------------------------------------------------------------

BATCH_CANDIDATES = (
    [{"delta": d, "relax_unroll": 2, "topup": 32} for d in (25000, 50000, 100000)]
    + [{"delta": 25000, "relax_unroll": 2, "topup": 16},
       {"delta": 50000, "relax_unroll": 4, "topup": 16}]
    + [{"delta": d, "relax_unroll": 2, "topup": 32, "light_heavy": 1, "bucket_sync": 1}
       for d in (25000, 50000)])


def batch_candidates():
    """BATCH_CANDIDATES plus the CTA count (work blocks): two or three CTAs
    per SM instead of the four that fit.  Queries on small graphs share one
    small frontier among a query's CTAs, and fewer CTAs per query contend
    less (64 queries on a 1024^2 grid: 19.7 ms at four per SM, 16.8 ms at
    two)."""
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    return list(BATCH_CANDIDATES) + [{"delta": 25000, "relax_unroll": 2, "topup": 16,
                                      "work_blocks": k * sms} for k in (2, 3)]


def batched_arm(args, rep, local):
    """C4: one step = one batched launch of all sources (CUDA-graph replay)."""
    import torch
    from mlmq_tpds_withl3_b200 import BatchSolver, DeviceGraph, Solver, autotune, default_config
    from mlmq_tpds_withl3_b200 import workloads
    from mlmq_tpds_withl3_b200.replicas import whole_job_rate
    ol = oracle_lib()
    side = args.side or (SMALL["c4_side"] if args.small else 4896)
    g, srcs = workloads.c4(side=side)
    if args.sources:
        srcs = srcs[:args.sources]
    dg = DeviceGraph.upload(g)
    queries = [(dg, s) for s in srcs]
    tune_report = None
    if args.no_tune:
        bcfg = default_config(delta=25000, warps_per_block=8, relax_unroll=2, topup=32,
                              l2_cap_log2=20, l2_batch=16, bucket_max=2)
    else:
        bcfg, tune_report = autotune.tune_batch(queries, dg.slots, candidates=batch_candidates())
    batch = BatchSolver(len(srcs), dg.slots + (dg.n if bcfg.light_heavy else 0), bcfg)
    stream = torch.cuda.Stream()

    # The back-to-back baseline gets its own tuned single-solve configuration,
    # picked on sources other than the timed ones.
    if args.no_tune:
        pcfg = default_config(delta=200000)
    else:
        probes = workloads.probe_sources(g, srcs, count=4, pool=np.arange(g.n))
        scratch = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        pcfg, _ = autotune.tune(dg, g, probes, kind="c4-plain", use_cache=False,
                                between=lambda: (scratch.zero_(), torch.cuda.synchronize()))
        del scratch
    plain = Solver(dg, pcfg)
    plain_ms, plain_out = [], []
    for s in srcs:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plain.launch(s, stream.cuda_stream)
        e1.record(stream)
        plain.wait()
        e1.synchronize()
        plain_ms.append(e0.elapsed_time(e1))
        plain_out.append(plain.dist())
    plain.close()

    for _ in range(args.warmup):
        batch.launch(queries, use_graph=True, stream=stream.cuda_stream)
        batch.wait()
    torch.cuda.synchronize()
    rep.barrier()
    events = []
    steps = max(1, args.batch_steps)
    sampler = ClockSampler(local)
    with sampler:
        for _ in range(steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.launch(queries, use_graph=True, stream=stream.cuda_stream)
            e1.record(stream)
            batch.wait()
            events.append((e0, e1))
        torch.cuda.synchronize()
    rep.barrier()
    step_ms = np.array([a.elapsed_time(b) for a, b in events])
    total_s = rep.max(step_ms.sum() / 1e3)

    # Every query of the last launch and every back-to-back solve against the
    # oracle, element by element (outside the timed region).
    t0 = time.perf_counter()
    ref, works = ol.sssp_many(g, srcs)
    correct = True
    reached = []
    for q in range(len(srcs)):
        d = batch.dist(q)
        correct = correct and np.array_equal(d, ref[q]) and np.array_equal(plain_out[q], ref[q])
        reached.append(int((ref[q] != ol.INT_MAX).sum()))
    check_s = time.perf_counter() - t0
    del ref, plain_out
    batch.close()
    dg.close()

    qps = whole_job_rate(len(srcs) * steps, rep.world, total_s)
    plain_qps = whole_job_rate(len(srcs), rep.world, rep.max(np.sum(plain_ms) / 1e3))
    work_step = float(np.sum(works))
    bytes_step = 12.0 * work_step + 12.0 * float(sum(reached))
    achieved = bytes_step * steps / total_s / 1e9
    peak, peak_kind = measured_peak()
    out = {
        "metric": BATCH_METRIC, "value": qps, "unit": "queries/s", "steps": steps,
        "warmup": args.warmup, "ms_per_step": total_s / steps * 1e3,
        "config": {"workload": WORKLOAD_TEXT["c4"] if side == 4896 else
                   f"batched: {len(srcs)} sources on a {side}x{side} grid (scaled down)",
                   "n": g.n, "m": g.m, "sources": len(srcs),
                   "graph_sha256_16": graph_digest(g),
                   "l2": "inputs (6.1 GB distances, 0.7 GB arcs) exceed L2"},
        "solver": {**cfg_summary(bcfg), "grid": batch.grid, "cuda_graph": True},
        "correct": bool(correct),
        "checked": f"all {len(srcs)} batched results and all {len(srcs)} back-to-back results "
                   f"element by element against the oracle ({check_s:.1f} s, untimed)",
        "gteps": work_step * steps / total_s / 1e9,
        "plain_back_to_back": {"qps": plain_qps, "ms_per_query_p50": float(np.median(plain_ms)),
                               "config": cfg_summary(pcfg),
                               "gteps": work_step / (np.sum(plain_ms) / 1e3) / 1e9},
        "speedup_vs_plain_qps": qps / plain_qps,
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                       "p99": float(np.percentile(step_ms, 99)),
                       "note": "every query of a batch completes within its launch"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": ncu_traffic("sssp_batch_kernel", "c4")[0],
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "kernel": "sssp_batch_kernel",
                     "algorithmic_bytes_per_launch": bytes_step},
        "clocks": sampler.summary(), "gpu_launches": len(events),
    }
    if tune_report:
        out["autotune"] = {"config": tune_report["config"], "trials": len(tune_report["trials"])}
    return out


# ---- served arm (C5) -----------------------------------------------------------------

SERVE_CANDIDATES = (
    [{"delta": d, "topup": 32} for d in (25000, 50000, 100000, 200000)]
    + [{"delta": 50000, "topup": 16}]
    + [{"delta": d, "topup": 32, "light_heavy": 1, "bucket_sync": 1} for d in (25000, 50000)])


def served_arm(args, rep, local):
    """C5: Poisson arrivals over 8 resident graphs: a run at the offered rate
    (latency) and a saturating burst (throughput); every result's device
    digest against the oracle's."""
    import torch
    from mlmq_tpds_withl3_b200 import DeviceGraph, Solver, autotune, default_config, workloads
    from mlmq_tpds_withl3_b200._lib import dist_digest
    from mlmq_tpds_withl3_b200.server import (HOST_TIMEOUT, PinnedPool, Server,
                                              poisson_schedule, serve_poisson, summarize)
    ol = oracle_lib()
    if args.small:
        hgs = workloads.c5_graphs(max_log2=SMALL["c5_max_log2"], rmat_scales=SMALL["c5_rmat"])
    else:
        hgs = workloads.c5_graphs()
    names = list(hgs)
    dgs = [DeviceGraph.upload(hgs[k]) for k in names]
    ns = [hgs[k].n for k in names]
    max_n = max(dg.slots for dg in dgs)
    # Vertices up to 1024 arcs are spread over the warp's lanes with the
    # others' arcs instead of being relaxed one at a time by the whole warp
    # (heavier ones are split into pieces anyway): R-MAT solves ran faster
    # that way, grids (degree <= 4) do not notice.
    cfg = default_config(delta=100000, warps_per_block=args.slot_warps, relax_unroll=2,
                         l2_cap_log2=20, l2_batch=16, bucket_max=2, large_degree=4096)
    knobs = None
    tune_report = None
    if not args.no_tune:
        # Each resident graph gets the per-query settings that were fastest on
        # a batched launch of 64 of its own queries (sources other than the
        # served ones); the server passes them with every query.
        knobs, tune_report = [], {}
        base = {**autotune.BATCH_BASE, "warps_per_block": args.slot_warps, "relax_unroll": 2,
                "large_degree": 4096}
        for i, dg in enumerate(dgs):
            rng = np.random.default_rng(70 + i)
            qs = [(dg, int(s)) for s in rng.integers(0, ns[i], 64)]
            kc, trep = autotune.tune_batch(qs, dg.slots, candidates=SERVE_CANDIDATES, base=base)
            knobs.append(kc)
            tune_report[names[i]] = dict(trep["config"])
        if any(k.light_heavy for k in knobs):
            max_n = max(max_n, max(dg.slots + dg.n for dg, k in zip(dgs, knobs)
                                   if k.light_heavy))
            for dg, k in zip(dgs, knobs):
                if k.light_heavy:
                    dg.prepare_light(k.delta)
    sv = Server(slots=args.slots, max_vertices=max_n, cfg=cfg, lifetime_s=900)
    pool = PinnedPool(sv.slots, max(ns))  # result buffers hold real vertices only
    runs = {}
    scheds = {}
    sampler = ClockSampler(local)
    with sampler:
        for key, rate, seed, count in (("light", args.light_rate, 100, args.light_queries),
                                       ("offered", args.served_rate, 101, args.served_queries),
                                       ("saturation", args.burst_rate, 102, args.served_queries)):
            sched = poisson_schedule(rate, count, ns, seed=seed)
            recs = serve_poisson(sv, dgs, sched, pool=pool, timeout_s=600, knobs=knobs)
            runs[key] = recs
            scheds[key] = sched
    clocks = sampler.summary()
    info = {"slots": sv.slots, "grid": sv.grid, "block": sv.block}
    sv.close()
    del pool

    # Back-to-back plain solves of a sample of the same mix, each graph with
    # its own tuned single-solve configuration; the same queries alone must
    # give the digest they had in the mix.
    sample = runs["saturation"][:96]
    scratch = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flush_l2():
        scratch.zero_()
        torch.cuda.synchronize()

    solvers = {}
    plain_ms, plain_by_graph = [], {}
    alone_same = True
    stream = torch.cuda.Stream()
    for r in sample:
        gi = r["graph"]
        if gi not in solvers:
            pc = default_config(delta=200000)
            if not args.no_tune:
                hg = hgs[names[gi]]
                served_srcs = [x["src"] for x in sample if x["graph"] == gi]
                probe = workloads.probe_sources(hg, served_srcs, count=4,
                                                pool=np.flatnonzero(np.diff(hg.row) > 0))
                pc, _ = autotune.tune(dgs[gi], hg, probe, kind=f"c5-{names[gi]}",
                                      use_cache=False, between=flush_l2)
            solvers[gi] = Solver(dgs[gi], pc)
        s = solvers[gi]
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.launch(r["src"], stream.cuda_stream)
        e1.record(stream)
        s.wait()
        e1.synchronize()
        plain_ms.append(e0.elapsed_time(e1))
        plain_by_graph.setdefault(names[gi], []).append(plain_ms[-1])
        if r["status"] != 0 or dist_digest(s.dist()) != r["digest"]:
            alone_same = False
    for s in solvers.values():
        s.close()
    for dg in dgs:
        dg.close()

    # Every served result against the oracle: digest of the oracle's
    # distances for each (graph, source) served.
    t0 = time.perf_counter()
    want = {}
    for gi, name in enumerate(names):
        srcs = sorted({r["src"] for recs in runs.values() for r in recs if r["graph"] == gi})
        if not srcs:
            continue
        dgst, _, _ = ol.sssp_digest_many(hgs[name], srcs)
        for s, d in zip(srcs, dgst):
            want[(gi, s)] = int(d)
    check_s = time.perf_counter() - t0
    bad = 0
    total = 0
    for recs in runs.values():
        for r in recs:
            total += 1
            if r["status"] != 0 or r["digest"] != want[(r["graph"], r["src"])]:
                bad += 1
    sat = summarize(runs["saturation"], names)
    off = summarize(runs["offered"], names)
    light = summarize(runs["light"], names)
    plain_qps = 1e3 / float(np.mean(plain_ms))
    qps = rep.sum(sat["qps"])
    plain_qps = rep.sum(plain_qps)
    out = {
        "metric": SERVE_METRIC, "value": qps, "unit": "queries/s",
        "config": {"workload": WORKLOAD_TEXT["c5"] + (" [scaled down]" if args.small else ""),
                   "graphs": {k: {"n": hgs[k].n, "m": hgs[k].m} for k in names},
                   "queries_per_run": args.served_queries,
                   "offered_rate": args.served_rate, "burst_rate": args.burst_rate,
                   "light_rate": args.light_rate, "light_queries": args.light_queries,
                   **info, "slot_settings": cfg_summary(cfg)},
        "saturation": {k: sat.get(k) for k in ("qps", "p50_ms", "p99_ms", "mean_ms", "finished",
                                               "errors", "error_codes")},
        "offered": {k: off.get(k) for k in ("qps", "p50_ms", "p99_ms", "mean_ms", "finished",
                                            "errors", "error_codes")},
        "light": {k: light.get(k) for k in ("qps", "p50_ms", "p99_ms", "mean_ms", "finished",
                                            "errors", "error_codes")},
        "latency_ms": {"p50": off["p50_ms"], "p99": off["p99_ms"],
                       "at_offered_rate": args.served_rate},
        "per_graph_saturation": sat.get("per_graph"),
        "plain_back_to_back": {"qps": plain_qps, "queries": len(plain_ms),
                               "ms_per_query_mean": float(np.mean(plain_ms)),
                               "ms_mean_by_graph": {k: float(np.mean(v))
                                                    for k, v in sorted(plain_by_graph.items())}},
        "speedup_vs_plain_qps": qps / plain_qps,
        "correct": bool(bad == 0 and alone_same),
        "checked": f"all {total} served results: status 0 and the device digest of each "
                   f"distance array equal to the digest of the oracle's distances "
                   f"({check_s:.1f} s, untimed); {len(sample)} of them also solved alone "
                   f"with the plain solver, same digest",
        "mismatches": bad, "alone_equals_mix": bool(alone_same),
        "clocks": clocks,
    }
    if tune_report:
        out["autotune"] = {"per_graph_query_settings": tune_report}
    del HOST_TIMEOUT
    return out


# ---- arms ------------------------------------------------------------------------------

def run_reference(args):
    """The reference's own sssp_sequential on the headline workload, one host
    thread per source; rank 0 only."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    name, g, srcs = reference_workload(args)
    threads = max(1, min(len(srcs), os.cpu_count() or 1))
    for _ in range(args.warmup):
        cpu_reference_gteps(g, srcs, threads)
    work = wall = 0.0
    kind = "reference"
    for _ in range(args.steps):
        w, t, _, kind = cpu_reference_gteps(g, srcs, threads)
        work += w
        wall += t
    gteps = work / wall / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": gteps, "unit": "GTEPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator; the reference's DIMACS graphs are not available)",
        "config": workload_config(name, g, srcs, args.small),
        "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": threads, "kind": kind,
                         "host_cpu": host_cpu(),
                         "sample": f"{len(srcs)} sources per step, one host thread each, "
                                   f"sssp_sequential (SS/SSSP/main.cu:47)"},
        "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_mlmq(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from mlmq_tpds_withl3_b200.replicas import Replicas
    from mlmq_tpds_withl3_b200._lib import lib
    rep = Replicas("nccl", timeout_s=1800)
    name, g, srcs = headline_workload(args)
    res = plain_arm(args, name, g, srcs, rep, local, args.steps, args.warmup,
                    cpu_baseline=not args.no_cpu_baseline, e2e_on=not args.no_e2e)
    del g
    lib.mlmq_release_cached()
    line = {"metric": METRIC, "value": res.pop("value"), "unit": res.pop("unit"),
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res.pop("ms_per_step"), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator; the reference's DIMACS graphs are not available)",
            "config": res.pop("config"), "parallelism": "replicas" if world > 1 else "single GPU"}
    res.pop("steps")
    res.pop("warmup")
    line.update(res)
    skip = {s.strip() for s in args.skip.split(",") if s.strip()}
    if args.workload == "all" and world == 1:
        blocks_t0 = time.perf_counter()
        if "c3" not in skip:
            from mlmq_tpds_withl3_b200 import workloads
            if args.small:
                g3, s3 = workloads.c3(scale=SMALL["c3_scale"])
            else:
                g3, s3 = workloads.c3()
            c3 = plain_arm(args, "c3", g3, s3, rep, local, min(args.steps, 10), args.warmup,
                           cpu_baseline=False, e2e_on=not args.no_e2e)
            c3["metric"] = "SSSP GTEPS (plain single-source, R-MAT scale 22)"
            line["c3"] = c3
            del g3
            lib.mlmq_release_cached()
        if "batched" not in skip:
            line["batched"] = batched_arm(args, rep, local)
            lib.mlmq_release_cached()
        if "served" not in skip:
            line["served"] = served_arm(args, rep, local)
            lib.mlmq_release_cached()
        line["blocks_wall_s"] = time.perf_counter() - blocks_t0
        line["correct_all"] = bool(line["correct"] and all(
            line[k]["correct"] for k in ("c3", "batched", "served") if k in line))
    rep.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_single_block(args, which):
    """--workload c4 or c5: that block alone as the JSON line."""
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from mlmq_tpds_withl3_b200.replicas import Replicas
    rep = Replicas("nccl", timeout_s=1800)
    res = batched_arm(args, rep, local) if which == "c4" else served_arm(args, rep, local)
    rep.close()
    line = {"metric": res.pop("metric"), "value": res.pop("value"), "unit": res.pop("unit"),
            "n_gpus": world, "steps": res.pop("steps", 1), "warmup": res.pop("warmup", 0),
            "ms_per_step": res.pop("ms_per_step", None), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generators)"}
    line.update(res)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload in ("c4", "c5"):
        return run_single_block(args, args.workload)
    return run_mlmq(args)


if __name__ == "__main__":
    sys.exit(main())
