"""B200-native (sm_100a) delta-stepping single-source shortest paths.

A from-scratch implementation of the MLMQ solver's hot path
(hideoze/mlmq_tpds_withl3): warp-private SLF L1 queues, HBM delta-bucket L2
queues, an in-device L3 overflow ring, persistent warps, CSR relaxation with
integer atomicMin and bounded-wait termination, all in libmlmq_b200.so.
"""
from ._lib import Config, GraphInfo, MlmqError, default_config, MLMQ_L1SLF_L2DQ, MLMQ_L1V_L2DQ
from .graph import HostGraph
from .solver import (DeviceGraph, Solver, solve_host, sssp_init, sssp_re_init,
                     sssp_run_adaptive, sssp_cp_data, INT_MAX)
from .batch import BatchSolver

__all__ = [
    "Config", "GraphInfo", "MlmqError", "default_config", "MLMQ_L1SLF_L2DQ", "MLMQ_L1V_L2DQ",
    "HostGraph", "DeviceGraph", "Solver", "solve_host", "sssp_init", "sssp_re_init",
    "sssp_run_adaptive", "sssp_cp_data", "INT_MAX", "BatchSolver",
]
