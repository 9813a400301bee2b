"""Batched multi-source solving: many queries in one persistent launch.

The reference answers several sources with back-to-back full solver runs
(SSSP/main.cu:213-307).  ``BatchSolver.run`` solves every (graph, source)
query of a batch in ONE launch: each query gets a slot (its own distance
array and queue rings) and a group of CTAs, and the graph arrays are shared.
With ``use_graph=True`` the launch is captured in a CUDA graph the first time
a query set is seen and replayed afterwards.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib


class BatchSolver:
    def __init__(self, max_queries, max_vertices, cfg=None):
        self._h = None
        if cfg is None or isinstance(cfg, dict):
            over = {"warps_per_block": 8, **(cfg or {})}
            cfg = _lib.default_config(**over)
        self.cfg = cfg
        self.max_queries = max_queries
        self.max_vertices = max_vertices
        h = ctypes.c_void_p()
        check(lib.mlmq_batch_create(max_queries, max_vertices, ctypes.byref(cfg),
                                    ctypes.byref(h)), "mlmq_batch_create")
        self._h = h
        self._graphs = []
        self._n = []
        grid, block, mq = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib.mlmq_batch_info(h, ctypes.byref(grid), ctypes.byref(block), ctypes.byref(mq)))
        self.grid, self.block = grid.value, block.value

    def close(self):
        if self._h is not None and self._h.value:
            lib.mlmq_batch_destroy(self._h)
        self._h = None

    __del__ = close

    def launch(self, queries, use_graph=False, stream=0):
        """queries: list of (DeviceGraph, source).  Enqueues one launch."""
        nq = len(queries)
        self._graphs = [g for g, _ in queries]  # keep the graphs alive
        self._n = [g.n for g, _ in queries]
        arr = (ctypes.c_void_p * nq)(*[g.handle.value for g, _ in queries])
        srcs = np.ascontiguousarray([s for _, s in queries], dtype=np.int32)
        self._srcs = srcs
        check(lib.mlmq_batch_run(self._h, nq, arr, srcs.ctypes.data, int(bool(use_graph)),
                                 ctypes.c_void_p(stream or None)), "mlmq_batch_run")

    def wait(self):
        check(lib.mlmq_batch_wait(self._h), "mlmq_batch_wait")

    def run(self, queries, use_graph=False):
        self.launch(queries, use_graph)
        self.wait()
        return self

    def dist(self, q):
        out = np.empty(self._n[q], dtype=np.int32)
        check(lib.mlmq_batch_copy_dist(self._h, q, out.ctypes.data), "mlmq_batch_copy_dist")
        return out

    def dist_ptr(self, q):
        p = ctypes.c_void_p()
        check(lib.mlmq_batch_dist(self._h, q, ctypes.byref(p)))
        return p.value

    def control(self, q, count=272):
        """Query q's control-block words when its last launch ended."""
        arr = (ctypes.c_uint32 * count)()
        check(lib.mlmq_batch_control(self._h, q, arr, count), "mlmq_batch_control")
        return np.frombuffer(arr, dtype=np.uint32).copy()

    def stats(self, q):
        st = _lib.SolveStats()
        status = ctypes.c_uint32()
        check(lib.mlmq_batch_query_status(self._h, q, ctypes.byref(status), ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in st._fields_}
