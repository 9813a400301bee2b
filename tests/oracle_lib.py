"""Test-side access to the CPU oracle (oracle/liboracle.so) and, when it was
built, the reference's own sssp_sequential (oracle/_ref/libref_sssp.so).

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_sssp.so")
INT_MAX = 2**31 - 1

_vp = ctypes.c_void_p
_oracle = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"{ORACLE_SO} missing: run `make -C oracle liboracle.so`")
        lib = ctypes.CDLL(ORACLE_SO)
        lib.oracle_sssp_i32.argtypes = [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp,
                                        ctypes.POINTER(ctypes.c_longlong)]
        lib.oracle_sssp_i64.argtypes = [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp,
                                        ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_longlong)]
        lib.oracle_sssp_many.argtypes = [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp, _vp,
                                         _vp, ctypes.c_int]
        for name in ("oracle_gen_grid", "oracle_gen_knn", "oracle_gen_rmat"):
            getattr(lib, name).restype = ctypes.c_int
        lib.oracle_free.argtypes = [_vp]
        lib.oracle_digest.argtypes = [ctypes.c_int, _vp]
        lib.oracle_digest.restype = ctypes.c_uint64
        lib.oracle_sssp_digest_many.argtypes = [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp,
                                                _vp, _vp, _vp, ctypes.c_int]
        _oracle = lib
    return _oracle


def reference():
    """The reference's compiled sssp_sequential, or None when not built."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        lib = ctypes.CDLL(REF_SO)
        lib.ref_sssp_sequential.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp,
                                            ctypes.c_int, _vp, ctypes.POINTER(ctypes.c_longlong)]
        _ref = lib
    return _ref


def _arr(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def sssp_i32(g, src):
    """oracle_sssp_i32 -> (dist, total_work)."""
    row, col, w = _arr(g.row), _arr(g.col), _arr(g.w)
    n = len(row) - 1
    d = np.empty(n, np.int32)
    work = ctypes.c_longlong()
    rc = oracle().oracle_sssp_i32(n, row.ctypes.data, col.ctypes.data, w.ctypes.data, int(src),
                                  d.ctypes.data, ctypes.byref(work))
    if rc:
        raise RuntimeError(f"oracle_sssp_i32 rc={rc}")
    return d, work.value


def sssp_i64(g, src):
    """oracle_sssp_i64 -> (dist, reached, max_dist)."""
    row, col, w = _arr(g.row), _arr(g.col), _arr(g.w)
    n = len(row) - 1
    d = np.empty(n, np.int32)
    reached = ctypes.c_int()
    mx = ctypes.c_longlong()
    rc = oracle().oracle_sssp_i64(n, row.ctypes.data, col.ctypes.data, w.ctypes.data, int(src),
                                  d.ctypes.data, ctypes.byref(reached), ctypes.byref(mx))
    if rc:
        raise RuntimeError(f"oracle_sssp_i64 rc={rc}")
    return d, reached.value, mx.value


def sssp_many(g, sources, threads=None):
    """Many sources on a thread pool -> (dist[nsrc, n], work[nsrc])."""
    row, col, w = _arr(g.row), _arr(g.col), _arr(g.w)
    n = len(row) - 1
    srcs = _arr(sources)
    d = np.empty((len(srcs), n), np.int32)
    work = np.empty(len(srcs), np.int64)
    threads = threads or os.cpu_count() or 1
    rc = oracle().oracle_sssp_many(n, row.ctypes.data, col.ctypes.data, w.ctypes.data,
                                   len(srcs), srcs.ctypes.data, d.ctypes.data, work.ctypes.data,
                                   int(threads))
    if rc:
        raise RuntimeError(f"oracle_sssp_many rc={rc}")
    return d, work


class CsrGraph:
    """A CSR graph held in numpy arrays (row n+1, col m, w m; int32)."""

    def __init__(self, row, col, w, name="graph"):
        self.row, self.col, self.w, self.name = row, col, w, name
        self.n = len(row) - 1
        self.m = len(col)


def _generated(fn, args, name):
    lib = oracle()
    n = ctypes.c_int()
    m = ctypes.c_longlong()
    row, col, w = _vp(), _vp(), _vp()
    rc = fn(*args, ctypes.byref(n), ctypes.byref(m), ctypes.byref(row), ctypes.byref(col),
            ctypes.byref(w))
    if rc:
        raise RuntimeError(f"{name} rc={rc}")
    try:
        take = lambda p, k: np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_int32)),
                                                  shape=(k,)).copy() if k else np.zeros(0, np.int32)
        return CsrGraph(take(row, n.value + 1), take(col, m.value), take(w, m.value), name)
    finally:
        for p in (row, col, w):
            lib.oracle_free(p)


def gen_grid(width, height, drop_p=0.10, wmin=1000, wmax=100000, seed=1):
    """oracle/workload.c's restatement of the road-like grid generator."""
    lib = oracle()
    return _generated(lib.oracle_gen_grid, (ctypes.c_int(width), ctypes.c_int(height),
                                            ctypes.c_double(drop_p), ctypes.c_int(wmin),
                                            ctypes.c_int(wmax), ctypes.c_uint64(seed)),
                      f"grid{width}x{height}")


def gen_knn(npoints, k=3, scale=1e6, seed=1):
    """oracle/workload.c's restatement of the planar kNN generator."""
    lib = oracle()
    return _generated(lib.oracle_gen_knn, (ctypes.c_int(npoints), ctypes.c_int(k),
                                           ctypes.c_double(scale), ctypes.c_uint64(seed)),
                      f"knn{npoints}k{k}")


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, wmin=1, wmax=1 << 20, seed=1):
    """oracle/workload.c's restatement of the R-MAT generator."""
    lib = oracle()
    return _generated(lib.oracle_gen_rmat, (ctypes.c_int(scale), ctypes.c_int(edge_factor),
                                            ctypes.c_double(a), ctypes.c_double(b),
                                            ctypes.c_double(c), ctypes.c_int(wmin),
                                            ctypes.c_int(wmax), ctypes.c_uint64(seed)),
                      f"rmat{scale}e{edge_factor}")


def digest(dist):
    """oracle_digest of an int32 distance array (the fingerprint the library's
    server reports for every served result)."""
    d = _arr(dist.numpy() if hasattr(dist, "numpy") else dist)
    return int(oracle().oracle_digest(len(d), d.ctypes.data))


def digest_numpy(dist):
    """The same fingerprint in numpy (an independent statement of it)."""
    d = np.ascontiguousarray(dist, dtype=np.int32)
    x = (np.arange(len(d), dtype=np.uint64) << np.uint64(32)) | d.view(np.uint32).astype(np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
        return int(np.sum(x, dtype=np.uint64))


def sssp_digest_many(g, sources, threads=None):
    """Many sources on a thread pool, keeping only each result's digest ->
    (digest[nsrc] uint64, work[nsrc], reached[nsrc])."""
    row, col, w = _arr(g.row), _arr(g.col), _arr(g.w)
    n = len(row) - 1
    srcs = _arr(sources)
    dg = np.empty(len(srcs), np.uint64)
    work = np.empty(len(srcs), np.int64)
    reached = np.empty(len(srcs), np.int32)
    threads = threads or os.cpu_count() or 1
    rc = oracle().oracle_sssp_digest_many(n, row.ctypes.data, col.ctypes.data, w.ctypes.data,
                                          len(srcs), srcs.ctypes.data, dg.ctypes.data,
                                          work.ctypes.data, reached.ctypes.data, int(threads))
    if rc:
        raise RuntimeError(f"oracle_sssp_digest_many rc={rc}")
    return dg, work, reached


def ref_sequential(g, src):
    """The reference's own sssp_sequential -> (dist, total_work)."""
    lib = reference()
    if lib is None:
        raise RuntimeError("oracle/_ref/libref_sssp.so not built")
    row, col, w = _arr(g.row), _arr(g.col), _arr(g.w)
    n = len(row) - 1
    d = np.empty(n, np.int32)
    work = ctypes.c_longlong()
    rc = lib.ref_sssp_sequential(n, len(col), row.ctypes.data, col.ctypes.data, w.ctypes.data,
                                 int(src), d.ctypes.data, ctypes.byref(work))
    if rc:
        raise RuntimeError(f"ref_sssp_sequential rc={rc}")
    return d, work.value


CHAIN_SO = os.path.join(ROOT, "oracle", "_ref", "libref_chain.so")
REORDER_BIN = os.path.join(ROOT, "oracle", "_ref", "reorder_gr")


def ref_chain_shortcuts(g, source, cut=None):
    """The reference's own chain-shortcut builder (SSSP/l3/l3_chain_shortcuts.h,
    compiled into oracle/_ref/libref_chain.so) -> (row, col, w, stats[5]), or
    None when that checker was not built."""
    if not os.path.exists(CHAIN_SO):
        return None
    lib = ctypes.CDLL(CHAIN_SO)
    lib.ref_chain_shortcuts.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int,
                                        ctypes.c_int, _vp, _vp, _vp, ctypes.c_longlong,
                                        ctypes.POINTER(ctypes.c_longlong), _vp]
    row, col, w = _arr(g.row), _arr(g.col), _arr(g.w)
    n = len(row) - 1
    cut = n if cut is None else cut
    cap = 2 * len(col) + 1
    orow = np.empty(n + 1, np.int32)
    ocol = np.empty(cap, np.int32)
    ow = np.empty(cap, np.int32)
    om = ctypes.c_longlong()
    st = np.zeros(5, np.int64)
    rc = lib.ref_chain_shortcuts(n, len(col), row.ctypes.data, col.ctypes.data, w.ctypes.data,
                                 int(cut), int(source), orow.ctypes.data, ocol.ctypes.data,
                                 ow.ctypes.data, cap, ctypes.byref(om), st.ctypes.data)
    if rc:
        raise RuntimeError(f"ref_chain_shortcuts rc={rc}")
    return orow, ocol[:om.value].copy(), ow[:om.value].copy(), st


def ref_reorder_bfs(gr_path, root, workdir):
    """Runs the reference's reorder_gr tool (oracle/_ref/reorder_gr) on a .gr
    file -> (out .gr path, perm, invperm), or None when it was not built."""
    if not os.path.exists(REORDER_BIN):
        return None
    import subprocess
    out = os.path.join(workdir, "reordered.gr")
    res = subprocess.run([REORDER_BIN, gr_path, out, str(int(root))], capture_output=True,
                         text=True)
    if res.returncode != 0:
        raise RuntimeError(f"reorder_gr failed: {res.stdout}{res.stderr}")
    perm = np.fromfile(out + ".perm.u32", dtype="<u4").astype(np.int32)
    inv = np.fromfile(out + ".invperm.u32", dtype="<u4").astype(np.int32)
    return out, perm, inv
