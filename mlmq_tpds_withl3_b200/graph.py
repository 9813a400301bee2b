"""Host graphs: seeded synthetic generators, .gr v1 I/O and the reference's
graph statistics.

All storage is owned by libmlmq_b200.so (``mlmq_host_graph``); the numpy
arrays exposed here are views valid for the lifetime of the HostGraph.
"""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import check, lib


def _view(ptr, count, dtype=np.int32):
    if count == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    buf = (ctypes.c_int32 * count).from_address(ptr)
    return np.frombuffer(buf, dtype=dtype, count=count)


class HostGraph:
    """A CSR graph in host memory: ``row`` (n+1), ``col`` (m), ``w`` (m), all
    int32; ``perm`` (n) for generators that reorder vertices, else None."""

    def __init__(self, handle, name="graph"):
        self._h = ctypes.c_void_p(handle)
        self.name = name
        n = ctypes.c_int()
        m = ctypes.c_int64()
        row, col, w, perm = (ctypes.c_void_p() for _ in range(4))
        check(lib.mlmq_hgraph_view(self._h, ctypes.byref(n), ctypes.byref(m),
                                   ctypes.byref(row), ctypes.byref(col),
                                   ctypes.byref(w), ctypes.byref(perm)), "view")
        self.n = n.value
        self.m = m.value
        self.row = _view(row.value, self.n + 1)
        self.col = _view(col.value, self.m)
        self.w = _view(w.value, self.m)
        self.perm = _view(perm.value, self.n) if perm.value else None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.mlmq_hgraph_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def __repr__(self):
        return f"HostGraph({self.name!r}, n={self.n}, m={self.m})"

    # ---- constructors ------------------------------------------------------
    @classmethod
    def grid(cls, width, height=None, drop_p=0.10, wmin=1000, wmax=100000, seed=1):
        """Road-like grid: 4-neighbour arcs, each undirected edge dropped with
        probability drop_p, one weight U{wmin..wmax} shared by both arcs."""
        height = width if height is None else height
        h = ctypes.c_void_p()
        check(lib.mlmq_hgraph_grid(width, height, drop_p, wmin, wmax, seed, ctypes.byref(h)),
              "mlmq_hgraph_grid")
        return cls(h.value, f"grid{width}x{height}")

    @classmethod
    def knn(cls, npoints, k=3, scale=1e6, seed=1):
        """Planar road-like graph: npoints uniform in the unit square, each
        joined to its k nearest neighbours (symmetrised), w=round(scale*d)+1."""
        h = ctypes.c_void_p()
        check(lib.mlmq_hgraph_knn(npoints, k, scale, seed, ctypes.byref(h)), "mlmq_hgraph_knn")
        return cls(h.value, f"knn{npoints}k{k}")

    @classmethod
    def rmat(cls, scale, edge_factor=16, a=0.57, b=0.19, c=0.19, wmin=1, wmax=1 << 20, seed=1):
        """R-MAT graph, directed, self-loops and duplicate arcs removed."""
        h = ctypes.c_void_p()
        check(lib.mlmq_hgraph_rmat(scale, edge_factor, a, b, c, wmin, wmax, seed,
                                   ctypes.byref(h)), "mlmq_hgraph_rmat")
        return cls(h.value, f"rmat{scale}e{edge_factor}")

    @classmethod
    def from_csr(cls, row, col, w, name="csr"):
        row = np.ascontiguousarray(row, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        w = np.ascontiguousarray(w, dtype=np.int32)
        n = len(row) - 1
        h = ctypes.c_void_p()
        check(lib.mlmq_hgraph_from_csr(n, len(col), row.ctypes.data, col.ctypes.data,
                                       w.ctypes.data, ctypes.byref(h)), "mlmq_hgraph_from_csr")
        return cls(h.value, name)

    @classmethod
    def read_gr(cls, path):
        """Galois/LonestarGPU .gr v1 (reference SSSP/csr_graph.cu:185-300)."""
        h = ctypes.c_void_p()
        check(lib.mlmq_hgraph_read_gr(os.fsencode(path), ctypes.byref(h)), f"read {path}")
        return cls(h.value, os.path.basename(str(path)))

    def write_gr(self, path):
        check(lib.mlmq_hgraph_write_gr(self._h, os.fsencode(path)), f"write {path}")

    # ---- transforms ----------------------------------------------------------
    def reorder_bfs(self, root=0):
        """BFS locality order (reference graph_transform/reorder_gr.cu:96-190).

        Returns (graph, perm, invperm): new ids follow the discovery order of
        a queue BFS from ``root`` that scans arcs in CSR order, unreached
        vertices follow in ascending id; perm[new] = old, invperm[old] = new.
        Distances carry over as dist_new[invperm[v]] == dist_old[v]."""
        h = ctypes.c_void_p()
        perm = np.empty(self.n, dtype=np.int32)
        inv = np.empty(self.n, dtype=np.int32)
        check(lib.mlmq_hgraph_reorder_bfs(self._h, int(root), ctypes.byref(h), perm.ctypes.data,
                                          inv.ctypes.data), "mlmq_hgraph_reorder_bfs")
        return HostGraph(h.value, f"{self.name}.bfs{root}"), perm, inv

    def reorder_bfs_gpu(self, root=0):
        """reorder_bfs computed on the current CUDA device
        (mlmq_hgraph_reorder_bfs_gpu); the same output."""
        h = ctypes.c_void_p()
        perm = np.empty(self.n, dtype=np.int32)
        inv = np.empty(self.n, dtype=np.int32)
        check(lib.mlmq_hgraph_reorder_bfs_gpu(self._h, int(root), ctypes.byref(h),
                                              perm.ctypes.data, inv.ctypes.data),
              "mlmq_hgraph_reorder_bfs_gpu")
        return HostGraph(h.value, f"{self.name}.bfs{root}"), perm, inv

    def chain_shortcuts(self, source=0, cut=None):
        """Chain-shortcut augmentation G+ (reference
        SSSP/l3/l3_chain_shortcuts.h:23-109): one extra arc per maximal walk
        through degree-2 chain vertices, every original arc kept, so all
        shortest-path distances are unchanged.  ``cut`` = n (default) places
        no partition restriction.  Returns (graph, stats)."""
        cut = self.n if cut is None else int(cut)
        h = ctypes.c_void_p()
        st = np.zeros(5, dtype=np.int64)
        check(lib.mlmq_hgraph_chain_shortcuts(self._h, cut, int(source), ctypes.byref(h),
                                              st.ctypes.data), "mlmq_hgraph_chain_shortcuts")
        keys = ("chain_vertices", "shortcuts", "longest_walk", "overflow_walks", "arcs_replaced")
        return HostGraph(h.value, f"{self.name}+"), dict(zip(keys, (int(x) for x in st)))

    # ---- statistics ----------------------------------------------------------
    def info(self):
        """The reference's graph_info (core/include/graph_info.h:24-67):
        degree and weight mean / max / population standard deviation."""
        deg = np.diff(self.row).astype(np.float64)
        gi = _lib.GraphInfo()
        gi.m, gi.nnz = self.n, self.m
        gi.avg_nnz = float(deg.mean()) if self.n else 0.0
        gi.max_nnz = float(deg.max()) if self.n else 0.0
        gi.dev_nnz = float(np.sqrt(((deg - gi.avg_nnz) ** 2).mean())) if self.n else 0.0
        wf = self.w.astype(np.float64)
        gi.avg_weight = float(wf.mean()) if self.m else 0.0
        gi.max_weight = float(wf.max()) if self.m else 0.0
        gi.dev_weight = float(np.sqrt(((wf - gi.avg_weight) ** 2).mean())) if self.m else 0.0
        gi.diameter = -1.0
        return gi

    def out_degree(self):
        return np.diff(self.row)
