"""Continuous-batching query server and a Poisson load generator.

``Server`` wraps mlmq_server_*: one persistent launch on the GPU serves
single-source queries on HBM-resident graphs while new ones arrive; each
query takes a free slot (a group of CTAs with its own distance array and
queues), runs alongside the other slots' queries, and its distances are
copied into a pinned host buffer when it finishes.

``serve_poisson`` drives a server with Poisson arrivals (each query picks a
graph uniformly and a source uniformly) and measures per-query latency
(finish - arrival, host clock) and throughput.
"""
import ctypes
import time
from collections import deque

import numpy as np

from . import _lib
from ._lib import MLMQ_ERR_BUSY, check, lib


class Server:
    """`slots` query slots of equal size, or `layout` = CTAs of each slot
    (small slots for latency-bound queries, wide ones for throughput-bound
    queries; a query's knobs.work_blocks asks for a slot of at least that
    many CTAs)."""

    def __init__(self, slots, max_vertices, cfg=None, lifetime_s=600.0, layout=None):
        if cfg is None or isinstance(cfg, dict):
            cfg = _lib.default_config(**{"warps_per_block": 8, **(cfg or {})})
        self.cfg = cfg
        h = ctypes.c_void_p()
        if layout is not None:
            arr = (ctypes.c_int * len(layout))(*layout)
            check(lib.mlmq_server_create_layout(len(layout), arr, max_vertices, ctypes.byref(cfg),
                                                int(lifetime_s * 1000), ctypes.byref(h)),
                  "mlmq_server_create_layout")
        else:
            check(lib.mlmq_server_create(slots, max_vertices, ctypes.byref(cfg),
                                         int(lifetime_s * 1000), ctypes.byref(h)),
                  "mlmq_server_create")
        self._h = h
        s, g, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib.mlmq_server_info(h, ctypes.byref(s), ctypes.byref(g), ctypes.byref(b)))
        self.slots, self.grid, self.block = s.value, g.value, b.value
        ctas = (ctypes.c_int * self.slots)()
        cnt = ctypes.c_int()
        check(lib.mlmq_server_layout(h, ctas, self.slots, ctypes.byref(cnt)))
        self.layout = list(ctas[:cnt.value])
        self.max_vertices = max_vertices
        self._tk = (ctypes.c_uint64 * 256)()
        self._st = (ctypes.c_int * 256)()
        self._ns = (ctypes.c_uint64 * 256)()
        self._res = (_lib.ServedResult * 256)()

    def submit(self, dgraph, src, out, knobs=None):
        """Returns a ticket, or None when every slot is busy.  `out` must be a
        host int32 buffer of dgraph.n entries (pinned for asynchronous copy)
        that stays alive until the ticket completes.  `knobs` (a Config)
        gives this query its own delta, topup, l1_ahead and bucket_max."""
        t = ctypes.c_uint64()
        ptr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
        if knobs is not None:
            rc = lib.mlmq_server_submit_cfg(self._h, dgraph.handle, int(src), ctypes.byref(knobs),
                                            ptr, ctypes.byref(t))
        else:
            rc = lib.mlmq_server_submit(self._h, dgraph.handle, int(src), ptr, ctypes.byref(t))
        if rc == MLMQ_ERR_BUSY:
            return None
        check(rc, "mlmq_server_submit")
        return t.value

    def poll(self):
        """[(ticket, status)] of queries whose distances are now on the host."""
        n = ctypes.c_int()
        check(lib.mlmq_server_poll(self._h, self._tk, self._st, 256, ctypes.byref(n)),
              "mlmq_server_poll")
        return [(self._tk[i], self._st[i]) for i in range(n.value)]

    def poll_timed(self):
        """[(ticket, status, solve_ms)]: as poll, with each query's device time
        from its slot taking the command to the slot reporting the result."""
        n = ctypes.c_int()
        check(lib.mlmq_server_poll_timed(self._h, self._tk, self._st, self._ns, 256,
                                         ctypes.byref(n)), "mlmq_server_poll_timed")
        return [(self._tk[i], self._st[i], self._ns[i] / 1e6) for i in range(n.value)]

    def poll_results(self):
        """[(ticket, status, solve_ms, digest)]: as poll_timed, with the
        device-computed digest of each result's distances
        (mlmq_dist_digest's definition; 0 for a failed query)."""
        n = ctypes.c_int()
        check(lib.mlmq_server_poll_results(self._h, self._res, 256, ctypes.byref(n)),
              "mlmq_server_poll_results")
        return [(r.ticket, r.status, r.solve_ns / 1e6, r.digest) for r in self._res[:n.value]]

    def busy(self):
        b = ctypes.c_int()
        rc = lib.mlmq_server_busy_slots(self._h, ctypes.byref(b))
        return b.value, rc == 0

    def close(self):
        if self._h is not None and self._h.value:
            lib.mlmq_server_destroy(self._h)
        self._h = None

    __del__ = close


class PinnedPool:
    """Pinned host buffers of `size` int32, one per in-flight query."""

    def __init__(self, count, size):
        import torch
        self.free = [torch.empty(size, dtype=torch.int32, pin_memory=True)
                     for _ in range(count)]

    def get(self):
        return self.free.pop() if self.free else None

    def put(self, buf):
        self.free.append(buf)


def poisson_schedule(rate, count, graphs_n, seed=1):
    """(arrival_s, graph_index, source) for `count` queries at `rate`/s."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=count))
    gi = rng.integers(0, len(graphs_n), size=count)
    src = [int(rng.integers(0, graphs_n[i])) for i in gi]
    return list(zip(t.tolist(), gi.tolist(), src))


HOST_TIMEOUT = "host_timeout"


def serve_poisson(server, dgraphs, schedule, keep=None, pool=None, timeout_s=300.0, knobs=None):
    """Runs the schedule against the server.  Returns a list of dicts
    (arrival, start, finish, latency_s, solve_ms, graph, src, status, digest
    [, dist]) in schedule order, digest being the device-computed result
    digest (None from a server without it); `keep(i)` selects the queries whose distances are kept;
    `knobs[graph index]` (optional) is that graph's per-query Config.

    A run that has not finished after `timeout_s` (host clock) stops there:
    queries still waiting or in flight get status HOST_TIMEOUT (and finish
    None) instead of an exception, so the caller sees every other query's
    status.  Queries still in flight keep their pinned buffers: close the
    server before reusing `pool`."""
    pool = pool or PinnedPool(server.slots, max(g.n for g in dgraphs))
    pending = deque(range(len(schedule)))
    inflight = {}
    out = [None] * len(schedule)
    t0 = time.perf_counter()
    while pending or inflight:
        now = time.perf_counter() - t0
        if now > timeout_s:
            for i, buf, start in list(inflight.values()) + [(i, None, None) for i in pending]:
                arr, gi, src = schedule[i]
                out[i] = {"arrival": arr, "start": start, "finish": None, "latency_s": None,
                          "solve_ms": None, "graph": gi, "src": src, "status": HOST_TIMEOUT,
                          "digest": None}
            break
        # Admit arrived queries in arrival order while slots and buffers are
        # free; a query whose slot size is all taken is passed over (it keeps
        # its place) so that it does not hold back queries that fit.
        # A slot class (the CTAs a query asks for) found full is not tried
        # again in this pass; a query that takes any slot finding none ends it.
        skipped = []
        full = set()
        while pending and schedule[pending[0]][0] <= now and len(skipped) < 256:
            i = pending[0]
            _, gi, src = schedule[i]
            kn = knobs[gi] if knobs is not None else None
            cls = kn.work_blocks if kn is not None else 0
            pending.popleft()
            if cls in full:
                skipped.append(i)
                continue
            buf = pool.get()
            if buf is None:
                skipped.append(i)
                break
            tk = server.submit(dgraphs[gi], src, buf, kn)
            if tk is None:
                pool.put(buf)
                skipped.append(i)
                full.add(cls)
                if cls == 0:
                    break
                continue
            inflight[tk] = (i, buf, now)
        pending.extendleft(reversed(skipped))
        done = (server.poll_results() if hasattr(server, "poll_results")
                else [(*x, None) for x in server.poll_timed()])
        for tk, status, solve_ms, digest in done:
            i, buf, start = inflight.pop(tk)
            arr, gi, src = schedule[i]
            fin = time.perf_counter() - t0
            rec = {"arrival": arr, "start": start, "finish": fin, "latency_s": fin - arr,
                   "solve_ms": solve_ms, "graph": gi, "src": src, "status": status,
                   "digest": digest}
            if keep is not None and keep(i):
                view = buf[:dgraphs[gi].n]  # a torch tensor or a numpy array
                rec["dist"] = (view.numpy() if hasattr(view, "numpy") else view).copy()
            out[i] = rec
            pool.put(buf)
        if not inflight and pending:
            wait = schedule[pending[0]][0] - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(min(wait, 0.001))
    return out


def summarize(records, names=None):
    """Throughput, latency percentiles and error counts of a served run;
    with `names` (graph index -> name) also per graph.  Throughput and
    latency count the queries that finished; every other status (device
    error codes and HOST_TIMEOUT) is counted in `error_codes`."""
    done = [r for r in records if r["finish"] is not None]
    codes = {}
    for r in records:
        if r["status"]:
            codes[str(r["status"])] = codes.get(str(r["status"]), 0) + 1
    out = {"queries": len(records), "finished": len(done), "errors": sum(codes.values()),
           "error_codes": codes}
    if done:
        lat = np.array([r["latency_s"] for r in done]) * 1e3
        span = max(r["finish"] for r in done) - min(r["arrival"] for r in done)
        out.update({"qps": len(done) / span, "p50_ms": float(np.percentile(lat, 50)),
                    "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean())})
    else:
        out.update({"qps": 0.0, "p50_ms": None, "p99_ms": None, "mean_ms": None})
    if names is not None:
        per = {}
        for gi, name in enumerate(names):
            sel = [r for r in done if r["graph"] == gi]
            if not sel:
                continue
            run = np.array([r["finish"] - r["start"] for r in sel]) * 1e3
            gl = np.array([r["latency_s"] for r in sel]) * 1e3
            per[name] = {"queries": len(sel), "errors": sum(1 for r in sel if r["status"]),
                         "p50_ms": float(np.percentile(gl, 50)),
                         "p99_ms": float(np.percentile(gl, 99)),
                         "run_ms_mean": float(run.mean()),
                         "solve_ms_mean": float(np.mean([r["solve_ms"] for r in sel]))}
        out["per_graph"] = per
    return out
