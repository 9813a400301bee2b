"""ctypes binding of libmlmq_b200.so (declared in include/mlmq_b200.h).

The shared library is built in-tree by ``make -C mlmq_tpds_withl3_b200`` (or
``__graft_entry__.build()``).  There is no fallback: importing this module
without the library raises ImportError.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmlmq_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing; build it with `make -C {_HERE}` "
        "(the SSSP solver has no CPU fallback)")

lib = ctypes.CDLL(LIB_PATH)

c_int = ctypes.c_int
c_i64 = ctypes.c_int64
c_u64 = ctypes.c_uint64
c_u32 = ctypes.c_uint32
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p
c_char_p = ctypes.c_char_p
P_int = ctypes.POINTER(ctypes.c_int)
PP_int = ctypes.POINTER(P_int)

MLMQ_OK = 0
ERRORS = {
    -1: "MLMQ_ERR_CUDA", -2: "MLMQ_ERR_ARG", -3: "MLMQ_ERR_TIMEOUT",
    -4: "MLMQ_ERR_QUEUE_FULL", -5: "MLMQ_ERR_STATE", -6: "MLMQ_ERR_NOMEM",
    -7: "MLMQ_ERR_UNSUPPORTED", -8: "MLMQ_ERR_RANGE", -9: "MLMQ_ERR_IO",
    -10: "MLMQ_ERR_NODEV", -11: "MLMQ_ERR_BUSY", -12: "MLMQ_ERR_MISMATCH",
}
globals().update({name: code for code, name in ERRORS.items()})

MLMQ_L1V_L2DQ = 0
MLMQ_L1SLF_L2DQ = 19


class MlmqError(RuntimeError):
    """A negative MLMQ_ERR_* return code from the library."""

    def __init__(self, code, what=""):
        self.code = code
        msg = lib.mlmq_strerror(code).decode()
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({msg})" if what else msg)


def check(code, what=""):
    if code != MLMQ_OK:
        raise MlmqError(code, what)
    return code


class Config(ctypes.Structure):
    """struct mlmq_config (include/mlmq_b200.h)."""
    _fields_ = [(n, c_int) for n in (
        "queue_type", "delta", "work_blocks", "warps_per_block", "l2_batch",
        "bucket_num", "bucket_max", "min_read", "large_degree", "l1_spill",
        "l2_cap_log2", "l3_cap_log2", "timeout_ms", "l1_keep", "relax_precheck",
        "relax_unroll", "l1_ahead", "topup", "bucket_sync", "light_heavy", "vertex_tiles")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class GraphInfo(ctypes.Structure):
    """struct graph_info (reference core/include/graph_info.h:8-22)."""
    _fields_ = [("m", c_int), ("nnz", c_int)] + [(n, ctypes.c_float) for n in (
        "avg_nnz", "max_nnz", "dev_nnz", "avg_weight", "dev_weight",
        "max_weight", "diameter")]


class SolveStats(ctypes.Structure):
    _fields_ = [("pushed", c_u64), ("l3_pushed", c_u64), ("relaxed", c_u64),
                ("improved", c_u64), ("first_max", c_u32), ("grid", c_int),
                ("block", c_int), ("status", c_u32), ("batches", c_u64), ("idle", c_u64)]


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("mlmq_strerror", c_char_p, c_int)
_sig("mlmq_config_default", c_int, ctypes.POINTER(Config))
# reference entry points (C linkage)
_sig("sssp_init", c_int, c_int, c_int, c_vp, c_vp, c_vp)
_sig("sssp_re_init", c_int)
_sig("sssp_run_adaptive", c_int, c_int, GraphInfo)
_sig("sssp_cp_data", c_int, PP_int)
# host graphs
_sig("mlmq_hgraph_grid", c_int, c_int, c_int, c_dbl, c_int, c_int, c_u64, ctypes.POINTER(c_vp))
_sig("mlmq_hgraph_knn", c_int, c_int, c_int, c_dbl, c_u64, ctypes.POINTER(c_vp))
_sig("mlmq_hgraph_rmat", c_int, c_int, c_int, c_dbl, c_dbl, c_dbl, c_int, c_int, c_u64,
     ctypes.POINTER(c_vp))
_sig("mlmq_hgraph_from_csr", c_int, c_int, c_i64, c_vp, c_vp, c_vp, ctypes.POINTER(c_vp))
_sig("mlmq_hgraph_read_gr", c_int, c_char_p, ctypes.POINTER(c_vp))
_sig("mlmq_hgraph_write_gr", c_int, c_vp, c_char_p)
_sig("mlmq_hgraph_view", c_int, c_vp, ctypes.POINTER(c_int), ctypes.POINTER(c_i64),
     ctypes.POINTER(c_vp), ctypes.POINTER(c_vp), ctypes.POINTER(c_vp), ctypes.POINTER(c_vp))
_sig("mlmq_hgraph_free", None, c_vp)
_sig("mlmq_hgraph_reorder_bfs", c_int, c_vp, c_int, ctypes.POINTER(c_vp), c_vp, c_vp)
_sig("mlmq_hgraph_chain_shortcuts", c_int, c_vp, c_int, c_int, ctypes.POINTER(c_vp), c_vp)
_sig("mlmq_hgraph_reorder_bfs_gpu", c_int, c_vp, c_int, ctypes.POINTER(c_vp), c_vp, c_vp)
_sig("mlmq_reorder_bfs_device", c_int, c_int, c_i64, c_vp, c_vp, c_vp, c_int, c_vp, c_vp, c_vp,
     c_vp, c_vp, c_vp)
# device graphs / solver
_sig("mlmq_graph_upload", c_int, c_int, c_i64, c_vp, c_vp, c_vp, ctypes.POINTER(c_vp))
_sig("mlmq_graph_wrap_device", c_int, c_int, c_i64, c_vp, c_vp, c_vp, ctypes.POINTER(c_vp))
_sig("mlmq_graph_size", c_int, c_vp, ctypes.POINTER(c_int), ctypes.POINTER(c_i64))
_sig("mlmq_graph_pieces", c_int, c_vp, ctypes.POINTER(c_int))
_sig("mlmq_graph_copy_arcs", c_int, c_vp, c_vp, c_vp)
_sig("mlmq_graph_prepare_light", c_int, c_vp, c_int)
_sig("mlmq_graph_prepare_tiles", c_int, c_vp, c_int)
_sig("mlmq_graph_free", None, c_vp)
_sig("mlmq_release_cached", c_int)
_sig("mlmq_solver_create", c_int, c_vp, ctypes.POINTER(Config), ctypes.POINTER(c_vp))
_sig("mlmq_solver_launch", c_int, c_vp, c_int, c_vp)
_sig("mlmq_solver_wait", c_int, c_vp)
_sig("mlmq_solver_solve", c_int, c_vp, c_int)
_sig("mlmq_solver_dist", c_int, c_vp, ctypes.POINTER(c_vp))
_sig("mlmq_solver_copy_dist", c_int, c_vp, c_vp)
_sig("mlmq_solver_stats", c_int, c_vp, ctypes.POINTER(SolveStats))
_sig("mlmq_solver_destroy", None, c_vp)
_sig("mlmq_solve_host", c_int, c_int, c_i64, c_vp, c_vp, c_vp, c_int, c_vp, c_vp,
     ctypes.POINTER(Config))
# batched multi-source solve
_sig("mlmq_batch_create", c_int, c_int, c_int, ctypes.POINTER(Config), ctypes.POINTER(c_vp))
_sig("mlmq_batch_info", c_int, c_vp, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
     ctypes.POINTER(c_int))
_sig("mlmq_batch_run", c_int, c_vp, c_int, ctypes.POINTER(c_vp), c_vp, c_int, c_vp)
_sig("mlmq_batch_wait", c_int, c_vp)
_sig("mlmq_batch_query_status", c_int, c_vp, c_int, ctypes.POINTER(c_u32),
     ctypes.POINTER(SolveStats))
_sig("mlmq_batch_dist", c_int, c_vp, c_int, ctypes.POINTER(c_vp))
_sig("mlmq_batch_control", c_int, c_vp, c_int, ctypes.POINTER(c_u32), c_int)
_sig("mlmq_batch_copy_dist", c_int, c_vp, c_int, c_vp)
_sig("mlmq_batch_destroy", None, c_vp)
# continuous-batching server
_sig("mlmq_server_create", c_int, c_int, c_int, ctypes.POINTER(Config), c_int,
     ctypes.POINTER(c_vp))
_sig("mlmq_server_create_layout", c_int, c_int, ctypes.POINTER(c_int), c_int, ctypes.POINTER(Config),
     c_int, ctypes.POINTER(c_vp))
_sig("mlmq_server_layout", c_int, c_vp, ctypes.POINTER(c_int), c_int, ctypes.POINTER(c_int))
_sig("mlmq_server_info", c_int, c_vp, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
     ctypes.POINTER(c_int))
_sig("mlmq_server_submit", c_int, c_vp, c_vp, c_int, c_vp, ctypes.POINTER(c_u64))
_sig("mlmq_server_submit_cfg", c_int, c_vp, c_vp, c_int, ctypes.POINTER(Config), c_vp,
     ctypes.POINTER(c_u64))
_sig("mlmq_server_poll", c_int, c_vp, ctypes.POINTER(c_u64), ctypes.POINTER(c_int), c_int,
     ctypes.POINTER(c_int))
_sig("mlmq_server_poll_timed", c_int, c_vp, ctypes.POINTER(c_u64), ctypes.POINTER(c_int),
     ctypes.POINTER(c_u64), c_int, ctypes.POINTER(c_int))
class ServedResult(ctypes.Structure):
    """struct mlmq_served_result."""
    _fields_ = [("ticket", c_u64), ("status", c_int), ("solve_ns", c_u64), ("digest", c_u64)]


_sig("mlmq_server_poll_results", c_int, c_vp, ctypes.POINTER(ServedResult), c_int,
     ctypes.POINTER(c_int))
_sig("mlmq_dist_digest", c_u64, c_vp, c_i64)
_sig("mlmq_server_busy_slots", c_int, c_vp, ctypes.POINTER(c_int))
_sig("mlmq_server_stop", c_int, c_vp)
_sig("mlmq_server_destroy", None, c_vp)
# single-source solve that allocates nothing (fixed workspace in the library)
_sig("mlmq_sssp_solve_noalloc", c_int, c_int, c_int, c_vp, c_vp, c_vp, c_int, c_vp,
     ctypes.POINTER(Config), c_vp)
NOALLOC_MAX_VERTICES = 1 << 20
NOALLOC_MAX_ARCS = 1 << 20


def dist_digest(dist):
    """mlmq_dist_digest of an int32 host array (numpy or a CPU torch tensor)."""
    import numpy as np
    a = dist.numpy() if hasattr(dist, "numpy") else dist
    a = np.ascontiguousarray(a, dtype=np.int32)
    return int(lib.mlmq_dist_digest(a.ctypes.data, len(a)))


def default_config(**overrides):
    """mlmq_config_default() (reference defaults + BENCH_DELTA/BENCH_QUEUE/
    MLMQ_WORK_BLOCKS), then keyword overrides."""
    cfg = Config()
    check(lib.mlmq_config_default(ctypes.byref(cfg)), "mlmq_config_default")
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, int(v))
    return cfg
