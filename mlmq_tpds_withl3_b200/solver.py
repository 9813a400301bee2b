"""Device graphs, the single-source solver and the reference's entry points.

The functions ``sssp_init``, ``sssp_re_init``, ``sssp_run_adaptive`` and
``sssp_cp_data`` keep the names, argument meaning and index conventions of the
reference solver (hideoze/mlmq_tpds_withl3,
evidence/l3_supplement_20260921_v2/single_source/SSSP/sssp_run.cu:676-976):
``sssp_init`` binds a DEVICE CSR (raw pointers), sources are 0-based and the
result is an int32 array with INT_MAX for unreachable vertices.  Errors raise
MlmqError instead of exiting the process.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib

INT_MAX = 2**31 - 1


class DeviceGraph:
    """A CSR graph resident on the current CUDA device."""

    def __init__(self, handle, n, m):
        self._h = ctypes.c_void_p(handle)
        self.n, self.m = n, m
        pc = ctypes.c_int()
        check(lib.mlmq_graph_pieces(self._h, ctypes.byref(pc)), "mlmq_graph_pieces")
        # vertex slots a batch or server needs for this graph: n plus the
        # pieces of its split heavy vertices
        self.pieces = pc.value
        self.slots = n + pc.value

    @classmethod
    def upload(cls, hg):
        """Copies a HostGraph (or anything with row/col/w numpy arrays)."""
        row = np.ascontiguousarray(hg.row, dtype=np.int32)
        col = np.ascontiguousarray(hg.col, dtype=np.int32)
        w = np.ascontiguousarray(hg.w, dtype=np.int32)
        n = len(row) - 1
        h = ctypes.c_void_p()
        check(lib.mlmq_graph_upload(n, len(col), row.ctypes.data, col.ctypes.data,
                                    w.ctypes.data, ctypes.byref(h)), "mlmq_graph_upload")
        return cls(h.value, n, len(col))

    @classmethod
    def wrap_device(cls, n, m, d_row, d_col, d_w):
        """Wraps caller-owned device arrays (integer device addresses)."""
        h = ctypes.c_void_p()
        check(lib.mlmq_graph_wrap_device(n, m, d_row, d_col, d_w, ctypes.byref(h)),
              "mlmq_graph_wrap_device")
        return cls(h.value, n, m)

    def prepare_light(self, delta):
        """Light-arc counts for the light/heavy split at this delta (needed
        before a server that runs light_heavy queries on this graph starts)."""
        check(lib.mlmq_graph_prepare_light(self._h, int(delta)), "mlmq_graph_prepare_light")

    def prepare_tiles(self, vertex_tiles):
        """The tile array of a vertex_tiles setting (2: 64-byte tiles with up
        to 8 inline arcs), needed before a server with that setting starts."""
        check(lib.mlmq_graph_prepare_tiles(self._h, int(vertex_tiles)), "mlmq_graph_prepare_tiles")

    def arcs(self):
        """(col, w): the arcs in the order the kernels read them -- each
        vertex's arcs a permutation of its input arcs, sorted by weight."""
        col = np.empty(self.m, np.int32)
        w = np.empty(self.m, np.int32)
        check(lib.mlmq_graph_copy_arcs(self._h, col.ctypes.data, w.ctypes.data),
              "mlmq_graph_copy_arcs")
        return col, w

    def close(self):
        if self._h is not None and self._h.value:
            lib.mlmq_graph_free(self._h)
        self._h = None

    __del__ = close

    @property
    def handle(self):
        return self._h


class Solver:
    """Single-source delta-stepping solver bound to one DeviceGraph.

    ``cfg`` is a ``_lib.Config`` or a dict of overrides of the defaults."""

    def __init__(self, dgraph, cfg=None):
        if cfg is None or isinstance(cfg, dict):
            cfg = _lib.default_config(**(cfg or {}))
        self.cfg = cfg
        self.graph = dgraph
        h = ctypes.c_void_p()
        check(lib.mlmq_solver_create(dgraph.handle, ctypes.byref(cfg), ctypes.byref(h)),
              "mlmq_solver_create")
        self._h = h

    def close(self):
        if self._h is not None and self._h.value:
            lib.mlmq_solver_destroy(self._h)
        self._h = None

    __del__ = close

    def launch(self, src, stream=0):
        """Enqueues one solve on a cudaStream_t handle (0: the solver's own)."""
        check(lib.mlmq_solver_launch(self._h, int(src), ctypes.c_void_p(stream or None)),
              "mlmq_solver_launch")

    def wait(self):
        check(lib.mlmq_solver_wait(self._h), "mlmq_solver_wait")

    def solve(self, src):
        check(lib.mlmq_solver_solve(self._h, int(src)), f"solve(src={src})")
        return self

    def dist_ptr(self):
        p = ctypes.c_void_p()
        check(lib.mlmq_solver_dist(self._h, ctypes.byref(p)), "mlmq_solver_dist")
        return p.value

    def dist(self, out=None):
        out = np.empty(self.graph.n, dtype=np.int32) if out is None else out
        check(lib.mlmq_solver_copy_dist(self._h, out.ctypes.data), "copy_dist")
        return out

    def stats(self):
        st = _lib.SolveStats()
        check(lib.mlmq_solver_stats(self._h, ctypes.byref(st)), "stats")
        return {n: getattr(st, n) for n, _ in st._fields_}


def solve_host(hg, sources, cfg=None):
    """The whole path with host buffers (mlmq_solve_host): upload, one solve
    per source, copy back.  Returns an (len(sources), n) int32 array."""
    if cfg is None or isinstance(cfg, dict):
        cfg = _lib.default_config(**(cfg or {}))
    srcs = np.ascontiguousarray(sources, dtype=np.int32)
    out = np.empty((len(srcs), hg.n), dtype=np.int32)
    check(lib.mlmq_solve_host(hg.n, hg.m, hg.row.ctypes.data, hg.col.ctypes.data,
                              hg.w.ctypes.data, len(srcs), srcs.ctypes.data, out.ctypes.data,
                              ctypes.byref(cfg)), "mlmq_solve_host")
    return out


# ---- reference entry points ---------------------------------------------------

_dropin_n = [0]  # vertex count bound by the last sssp_init


def sssp_init(m, nnz, RowPtr, ColIdx, edge_data):
    """sssp_run.cu:676 -- m vertices, nnz arcs; RowPtr/ColIdx/edge_data are
    device addresses (ints) of int32 arrays owned by the caller."""
    check(lib.sssp_init(int(m), int(nnz), RowPtr, ColIdx, edge_data), "sssp_init")
    _dropin_n[0] = int(m)
    return 0


def sssp_re_init():
    """sssp_run.cu:709 -- reset every distance to INT_MAX."""
    check(lib.sssp_re_init(), "sssp_re_init")
    return 0


def sssp_run_adaptive(src, info=None):
    """sssp_run.cu:888 -- solve from 0-based src (BENCH_WARMUPS/BENCH_REPEATS
    solves, one BENCH line each, as the reference)."""
    check(lib.sssp_run_adaptive(int(src), info if info is not None else _lib.GraphInfo()),
          "sssp_run_adaptive")
    return 0


def sssp_cp_data():
    """sssp_run.cu:749 -- the m distances as a numpy int32 array."""
    p = _lib.P_int()
    check(lib.sssp_cp_data(ctypes.byref(p)), "sssp_cp_data")
    try:
        n = _dropin_n[0]
        return np.ctypeslib.as_array(p, shape=(n,)).copy()
    finally:
        _libc.free(p)


_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]
_libc.free.restype = None
