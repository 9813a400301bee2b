#!/usr/bin/env python3
"""Benchmark of the plain single-source delta-stepping solve on B200.

Default workload (N=1): the planar road-like kNN graph -- 6.3M points uniform
in the unit square, 3 nearest neighbours symmetrised, w = round(1e6*d)+1 --
with 5 seeded sources solved one at a time and delta autotuned around
200000.  One step = those 5 solves.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mlmq|reference]
                  [--workload c1|c2|c3] [--sources S]

* value: GTEPS = sum of arcs out of reached vertices (the oracle's
  total_work) / summed device time of the solves, CUDA events on the launch
  stream, inputs resident in HBM, L2 flushed (256 MiB write) between solves.
* e2e: the same metric through mlmq_solve_host() with pinned host buffers:
  CSR upload, every solve, every distance copy back.
* roofline: algorithmic bytes per solve 12*m_r + 12*n_r over the kernel's
  average duration, against the measured HBM copy bandwidth.
* cpu_baseline: the reference's own sssp_sequential (oracle/_ref) -- or the
  oracle port when it was not built -- on the host, one thread.
* --impl reference: the reference's CPU implementation alone, one thread per
  source, on the same workload and metric.

Multi-GPU (torchrun): replicas only -- every rank solves the same job on its
own GPU with no collective on the data path; time is the max over ranks.
"""
import argparse
import csv
import io
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SSSP GTEPS (plain single-source delta-stepping, queries one at a time)"
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
}
BATCH_METRIC = "SSSP queries/sec (batched: 64 sources in one persistent launch)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("mlmq", "reference"), default="mlmq")
    ap.add_argument("--workload", choices=("c1", "c2", "c3", "c4", "c5"), default="c2")
    ap.add_argument("--rates", default="10,100,1000,5000", help="served: arrival rates /s")
    ap.add_argument("--serve-seconds", type=float, default=3.0)
    ap.add_argument("--max-queries", type=int, default=4000)
    ap.add_argument("--slots", type=int, default=64)
    ap.add_argument("--wide-slots", type=int, default=0,
                    help="served: wide slots for throughput-bound graphs (0: all slots equal; "
                         "on the 8-graph mix equal slots measured best)")
    ap.add_argument("--wide-ctas", type=int, default=54, help="served: CTAs of a wide slot")
    ap.add_argument("--slot-warps", type=int, default=8, help="served: worker warps per CTA")
    ap.add_argument("--sources", type=int, default=0, help="limit the number of sources")
    ap.add_argument("--side", type=int, default=0,
                    help="c4: grid side instead of 4896 (small cases for profiler captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--config", default="",
                    help="c1-c3: JSON overrides of the solver configuration, used instead of "
                         "tuning (reproducible profiler runs)")
    return ap.parse_args()


def load_workload(name, limit):
    from mlmq_tpds_withl3_b200 import workloads
    g, srcs = workloads.WORKLOADS[name]()
    if limit:
        srcs = srcs[:limit]
    return g, srcs


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kernel, workload):
    """Per-launch DRAM bytes from the committed ncu summary, if captured."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
                    return float(parts[2])
    except OSError:
        pass
    return None


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


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_gteps(g, srcs, threads):
    """Times the reference's sssp_sequential (or the oracle port) on the host."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    fn = oracle_lib.ref_sequential if oracle_lib.reference() is not None else oracle_lib.sssp_i32
    kind = "reference" if oracle_lib.reference() is not None else "port"

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


def run_reference(args):
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return 0
    g, srcs = load_workload(args.workload, args.sources)
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
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOAD_TEXT[args.workload], "n": g.n, "m": g.m,
                   "sources": srcs},
        "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": threads, "kind": kind,
                         "sample": f"{len(srcs)} sources per step, one host thread each, "
                                   f"sssp_sequential (SS/SSSP/main.cu:47)"},
        "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_mlmq(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    from mlmq_tpds_withl3_b200.replicas import Replicas, whole_job_rate
    rep = Replicas("nccl")
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    from mlmq_tpds_withl3_b200 import DeviceGraph, Solver, autotune, default_config
    from mlmq_tpds_withl3_b200._lib import check, lib

    g, srcs = load_workload(args.workload, args.sources)
    dg = DeviceGraph.upload(g)
    tune_report = None
    if args.config:
        cfg = default_config(**{"delta": 200000, **json.loads(args.config)})
    elif args.workload == "c1" or args.no_tune:
        cfg = default_config(delta=200000)
    else:
        cfg, tune_report = autotune.tune(dg, g, srcs[:2], kind=args.workload, use_cache=False)
    solver = Solver(dg, cfg)

    # Correctness and per-query work (oracle, untimed).
    dists, works = oracle_lib.sssp_many(g, srcs, threads=min(len(srcs), os.cpu_count() or 1))
    reached = (dists != oracle_lib.INT_MAX).sum(axis=1)
    correct = True
    for k, s in enumerate(srcs):
        solver.solve(s)
        if not np.array_equal(solver.dist(), dists[k]):
            correct = False

    stream = torch.cuda.Stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

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

    for _ in range(args.warmup):
        step(None)
    torch.cuda.synchronize()
    rep.barrier()
    events = []
    sampler = ClockSampler(local)
    with sampler:
        t_wall0 = time.perf_counter()
        for _ in range(args.steps):
            step(events)
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall0
    rep.barrier()
    per_query_ms = np.array([a.elapsed_time(b) for a, b in events])
    total_s = rep.max(per_query_ms.sum() / 1e3)
    work_step = float(np.sum(works))
    gteps = whole_job_rate(work_step * args.steps, world, total_s) / 1e9

    # Roofline of the persistent kernel.
    bytes_q = 12.0 * np.asarray(works, np.float64) + 12.0 * reached.astype(np.float64)
    launch_s = per_query_ms / 1e3
    achieved_gbs = float(np.sum(np.tile(bytes_q, args.steps)) / np.sum(launch_s) / 1e9)
    peak, peak_kind = measured_peak()
    traffic = ncu_traffic("sssp_plain_kernel", args.workload)

    # End to end through the host-buffer API.
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        row, col, w = pin(g.row), pin(g.col), pin(g.w)
        src_arr = np.asarray(srcs, np.int32)
        out = torch.empty((len(srcs), g.n), dtype=torch.int32).pin_memory()
        e2e_steps = max(1, min(args.steps, 5))
        walls = []
        for i in range(e2e_steps + 1):
            t0 = time.perf_counter()
            check(lib.mlmq_solve_host(g.n, g.m, row.data_ptr(), col.data_ptr(), w.data_ptr(),
                                      len(srcs), src_arr.ctypes.data, out.data_ptr(), cfg),
                  "mlmq_solve_host")
            if i:
                walls.append(time.perf_counter() - t0)
        e2e_s = rep.max(float(np.sum(walls)))
        correct = correct and np.array_equal(out.numpy(), dists)
        e2e = {"value": whole_job_rate(work_step * len(walls), world, e2e_s) / 1e9, "unit": "GTEPS",
               "h2d_bytes_per_step": int(4 * (g.n + 1) + 8 * g.m),
               "d2h_bytes_per_step": int(4 * g.n * len(srcs)),
               "ms_per_step": e2e_s / len(walls) * 1e3,
               "walls_ms": [round(x * 1e3, 2) for x in walls],
               "api": "mlmq_solve_host (pinned host CSR in, distances out)"}
    del dists

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        work, wall, busy, kind = cpu_reference_gteps(g, srcs, 1)
        cpu = {"value": work / wall / 1e9, "unit": "GTEPS", "cores": 1, "kind": kind,
               "sample": f"{len(srcs)} sources of the same workload, one after another, "
                         f"{wall:.1f} s"}

    rep.close()
    if rank != 0:
        return 0
    clocks = sampler.summary()
    line = {
        "metric": METRIC, "value": gteps, "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_s / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator; the reference's DIMACS graphs are not available)",
        "config": {"workload": WORKLOAD_TEXT[args.workload], "n": g.n, "m": g.m,
                   "sources": srcs, "queue": "L1SLF_L2DQ" if cfg.queue_type == 19 else "L1V_L2DQ",
                   "delta": cfg.delta, "warps_per_block": cfg.warps_per_block,
                   "work_blocks": solver.stats()["grid"],
                   "l2_between_solves": "flushed (256 MiB write, outside the timed events)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "correct": bool(correct),
        "qps": whole_job_rate(len(srcs) * args.steps, world, total_s),
        "latency_ms": {"p50": float(np.percentile(per_query_ms, 50)),
                       "p99": float(np.percentile(per_query_ms, 99))},
        "work_per_step": int(work_step),
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "kernel": "sssp_plain_kernel",
                     "algorithmic_bytes_per_launch": float(np.mean(bytes_q))},
        "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks,
        "gpu_launches": len(events), "wall_s_timed_region": t_wall,
    }
    if tune_report:
        line["autotune"] = {"config": tune_report.get("config"),
                            "trials": len(tune_report.get("trials", []))}
    print(json.dumps(line), flush=True)
    return 0


def run_batched(args):
    """C4: one step = one batched launch of all sources (CUDA-graph replay)."""
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    from mlmq_tpds_withl3_b200.replicas import Replicas, whole_job_rate
    rep = Replicas("nccl")
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    from mlmq_tpds_withl3_b200 import BatchSolver, DeviceGraph, Solver, default_config

    from mlmq_tpds_withl3_b200 import workloads
    g, srcs = workloads.c4(side=args.side) if args.side else workloads.c4()
    if args.sources:
        srcs = srcs[:args.sources]
    dg = DeviceGraph.upload(g)
    queries = [(dg, s) for s in srcs]
    tune_report = None
    if args.no_tune:
        # the configuration the batch tuner settles on for grids
        bcfg = default_config(delta=25000, warps_per_block=8, relax_unroll=2, topup=32,
                              l2_cap_log2=20, l2_batch=16, bucket_max=2)
    else:
        from mlmq_tpds_withl3_b200 import autotune
        bcfg, tune_report = autotune.tune_batch(queries, dg.slots)
    batch = BatchSolver(len(srcs), dg.slots + (dg.n if bcfg.light_heavy else 0), bcfg)
    stream = torch.cuda.Stream()

    # Correctness: oracle on a few sources, the plain solver on every source.
    check_q = list(range(0, len(srcs), max(1, len(srcs) // 4)))[:4]
    ref, works_chk = oracle_lib.sssp_many(g, [srcs[q] for q in check_q])
    batch.run(queries, use_graph=True)
    correct = all(np.array_equal(batch.dist(q), ref[i]) for i, q in enumerate(check_q))
    del ref
    # The back-to-back baseline gets its own tuned single-solve configuration.
    if args.no_tune:
        pcfg = default_config(delta=200000)
    else:
        from mlmq_tpds_withl3_b200 import autotune
        pcfg, _ = autotune.tune(dg, g, srcs[:2], kind="c4-plain", use_cache=False)
    plain = Solver(dg, pcfg)
    plain_ms, works, reached = [], [], []
    for q, s in enumerate(srcs):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plain.launch(s, stream.cuda_stream)
        e1.record(stream)
        plain.wait()
        e1.synchronize()
        plain_ms.append(e0.elapsed_time(e1))
        d = plain.dist()
        correct = correct and np.array_equal(d, batch.dist(q))
        fin = d != oracle_lib.INT_MAX
        reached.append(int(fin.sum()))
        works.append(int(np.diff(g.row)[fin].sum()))
    plain.close()
    work_step = float(sum(works))

    for _ in range(args.warmup):
        batch.launch(queries, use_graph=True, stream=stream.cuda_stream)
        batch.wait()
    torch.cuda.synchronize()
    rep.barrier()
    events = []
    sampler = ClockSampler(local)
    with sampler:
        for _ in range(args.steps):
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
    qps = whole_job_rate(len(srcs) * args.steps, world, total_s)
    plain_qps = whole_job_rate(len(srcs), world, rep.max(np.sum(plain_ms) / 1e3))
    rep.close()
    bytes_step = 12.0 * work_step + 12.0 * float(sum(reached))
    achieved = bytes_step * args.steps / total_s / 1e9
    peak, peak_kind = measured_peak()
    line = {
        "metric": BATCH_METRIC, "value": qps, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_s / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator)",
        "config": {"workload": WORKLOAD_TEXT["c4"] if not args.side else
                   f"batched: {len(srcs)} sources on a {args.side}x{args.side} grid (profiling case)",
                   "n": g.n, "m": g.m, "sources": len(srcs),
                   "delta": bcfg.delta, "warps_per_block": bcfg.warps_per_block,
                   "l1_ahead": bcfg.l1_ahead, "relax_unroll": bcfg.relax_unroll,
                   "grid": batch.grid,
                   "cuda_graph": True, "l2": "inputs (6.1 GB distances, 0.7 GB arcs) exceed L2"},
        "correct": bool(correct),
        "gteps": work_step * args.steps / total_s / 1e9,
        "plain_back_to_back": {"qps": plain_qps, "ms_per_query_p50": float(np.median(plain_ms)),
                               "config": {"delta": pcfg.delta, "warps_per_block": pcfg.warps_per_block,
                                          "relax_unroll": pcfg.relax_unroll,
                                          "l1_ahead": pcfg.l1_ahead,
                                          "vertex_tiles": pcfg.vertex_tiles},
                               "gteps": work_step / (np.sum(plain_ms) / 1e3) / 1e9},
        "speedup_vs_plain_qps": qps / plain_qps,
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                       "p99": float(np.percentile(step_ms, 99)),
                       "note": "every query of a batch completes within its launch"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": ncu_traffic("sssp_batch_kernel", "c4"),
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "kernel": "sssp_batch_kernel",
                     "algorithmic_bytes_per_launch": bytes_step},
        "clocks": sampler.summary(), "gpu_launches": len(events),
    }
    if tune_report:
        line["autotune"] = {"config": tune_report["config"], "trials": len(tune_report["trials"])}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


SERVE_METRIC = "SSSP queries/sec (served: continuous batching over 8 HBM-resident graphs)"


def run_served(args):
    """C5: Poisson arrivals over 8 resident graphs, rate swept 10..5000/s."""
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    from mlmq_tpds_withl3_b200.replicas import Replicas
    rep = Replicas("nccl", timeout_s=1800)
    from mlmq_tpds_withl3_b200 import DeviceGraph, Solver, default_config, workloads
    from mlmq_tpds_withl3_b200.server import (PinnedPool, Server, poisson_schedule,
                                              serve_poisson, summarize)
    hgs = workloads.c5_graphs()
    names = list(hgs)
    dgs = [DeviceGraph.upload(hgs[k]) for k in names]
    ns = [hgs[k].n for k in names]
    max_n = max(dg.slots for dg in dgs)
    tune_report = None
    cfg = default_config(delta=100000, warps_per_block=args.slot_warps, relax_unroll=2,
                         l2_cap_log2=20, l2_batch=16, bucket_max=2)
    knobs = None
    layout = None
    grid_max = 3 * 148  # CTAs of 8+1 warps that fit a B200 (the server checks)
    if args.wide_slots > 0:
        small = (grid_max - args.wide_slots * args.wide_ctas) // 6
        layout = [6] * small + [args.wide_ctas] * args.wide_slots
    if not args.no_tune:
        # Each resident graph gets the per-query settings (delta, topup,
        # run-ahead bound) that were fastest on a batched launch of 64 of its
        # own queries in small slots, and is sent to a wide slot when 8 of its
        # queries in wide slots give more queries/s than that (a
        # throughput-bound query gains nothing from sharing the GPU in small
        # pieces).  The server passes the settings with every query.
        from mlmq_tpds_withl3_b200 import autotune
        cands = [{"delta": d, "topup": t} for d in (25000, 50000, 100000, 200000)
                 for t in (16, 32)]
        cands += [{"delta": 400000, "topup": 16}, {"delta": 200000, "topup": 16, "l1_ahead": 0}]
        cands += [{"delta": d, "topup": 32, "light_heavy": 1, "bucket_sync": 1}
                  for d in (25000, 50000, 100000)]
        knobs, tune_report = [], {}
        base = {**autotune.BATCH_BASE, "warps_per_block": args.slot_warps, "relax_unroll": 2}
        for i, dg in enumerate(dgs):
            rng = np.random.default_rng(70 + i)
            qs = [(dg, int(s)) for s in rng.integers(0, ns[i], 64)]
            kc, trep = autotune.tune_batch(qs, dg.slots, candidates=cands, base=base)
            entry = dict(trep["config"])
            if layout is not None:
                qps_small = len(qs) / trep["seconds"]
                kw, repw = autotune.tune_batch(
                    qs[:8], dg.slots, candidates=cands,
                    base={**base, "work_blocks": 8 * args.wide_ctas})
                qps_wide = 8 / repw["seconds"]
                entry["qps_small_slots"] = qps_small
                entry["qps_wide_slots"] = qps_wide
                if qps_wide > qps_small:
                    kc = default_config(**{**base, **repw["config"], "work_blocks": args.wide_ctas})
                    entry = {**repw["config"], "work_blocks": args.wide_ctas,
                             "qps_small_slots": qps_small, "qps_wide_slots": qps_wide}
            knobs.append(kc)
            tune_report[names[i]] = entry
    if knobs is not None and any(k.light_heavy for k in knobs):
        max_n = max(max_n, max(dg.slots + dg.n for dg, k in zip(dgs, knobs) if k.light_heavy))
        for dg, k in zip(dgs, knobs):
            if k.light_heavy:
                dg.prepare_light(k.delta)
    sv = Server(slots=args.slots, max_vertices=max_n, cfg=cfg, lifetime_s=900, layout=layout)
    pool = PinnedPool(sv.slots, max(ns))  # result buffers hold real vertices only
    rates = [float(r) for r in args.rates.split(",")]
    sweep = []
    sample = {}
    for ri, rate in enumerate(rates):
        count = int(min(max(30, rate * args.serve_seconds), args.max_queries))
        sched = poisson_schedule(rate, count, ns, seed=100 + ri)
        # A kept result is copied out of its pinned buffer inside the serving
        # loop (up to 67 MB); eight per rate keep that host work small.
        every = max(1, count // 8)
        keep = (lambda i, every=every: i % every == 0)
        recs = serve_poisson(sv, dgs, sched, keep=keep, pool=pool, timeout_s=600, knobs=knobs)
        s = summarize(recs, names)
        s["rate"] = rate
        sweep.append(s)
        for i, r in enumerate(recs):
            if "dist" in r:
                sample[(ri, i)] = r
    sv.close()
    del pool
    # Alone vs in the mix, and back-to-back plain solves of the same mix.
    solvers = {}
    correct = True
    plain_ms = []
    plain_by_graph = {}
    stream = torch.cuda.Stream()
    for (ri, i), r in sample.items():
        gi = r["graph"]
        if gi not in solvers:
            # Each graph's back-to-back baseline runs its own tuned
            # single-solve configuration.
            pc = default_config(delta=200000)
            if not args.no_tune:
                from mlmq_tpds_withl3_b200 import autotune
                hg = hgs[names[gi]]
                probe = [int(x) for x in np.random.default_rng(gi).integers(0, hg.n, 2)]
                pc, _ = autotune.tune(dgs[gi], hg, probe, kind=f"c5-{names[gi]}", use_cache=False)
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
        if r["status"] or not np.array_equal(s.dist(), r["dist"]):
            correct = False
    for s in solvers.values():
        s.close()
    plain_qps = 1e3 / float(np.mean(plain_ms))
    top = max(sweep, key=lambda s: s["qps"])
    # replicas serve independent arrival streams: the whole job's rate is the
    # sum of theirs (one sum per collective, same order on every rank)
    top_qps = rep.sum(top["qps"])
    plain_qps = rep.sum(plain_qps)
    rep.close()
    line = {
        "metric": SERVE_METRIC, "value": top_qps, "unit": "queries/s", "n_gpus": world,
        "steps": len(rates), "warmup": 0, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generators)",
        "config": {"workload": "served: grids 2^16..2^24 + R-MAT 18/20/22 resident; Poisson "
                               "arrivals, graph and source uniform per query",
                   "graphs": {k: {"n": hgs[k].n, "m": hgs[k].m} for k in names},
                   "slots": sv.slots, "grid": sv.grid, "delta": cfg.delta,
                   "slot_ctas": sorted(set(sv.layout)) if layout else None,
                   "wide_slots": args.wide_slots if layout else 0,
                   "warps_per_block": cfg.warps_per_block, "relax_unroll": cfg.relax_unroll,
                   "l1_ahead": cfg.l1_ahead, "rates": rates},
        "sweep": sweep,
        "latency_ms": {"p50": top["p50_ms"], "p99": top["p99_ms"], "at_rate": top["rate"]},
        "plain_back_to_back": {"qps": plain_qps, "queries": len(plain_ms),
                               "ms_per_query_mean": float(np.mean(plain_ms)),
                               "ms_mean_by_graph": {k: float(np.mean(v))
                                                    for k, v in sorted(plain_by_graph.items())}},
        "speedup_vs_plain_qps": top_qps / plain_qps,
        "correct": bool(correct),
        "checked_alone_vs_mix": len(sample),
    }
    if tune_report:
        line["autotune"] = {"per_graph_query_settings": tune_report}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "c4":
        return run_batched(args)
    if args.workload == "c5":
        return run_served(args)
    return run_mlmq(args)


if __name__ == "__main__":
    sys.exit(main())
