"""The C-ABI library loads and exports every entry point the headers declare
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

import mlmq_tpds_withl3_b200 as mlmq
from mlmq_tpds_withl3_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions(header):
    text = open(os.path.join(INCLUDE, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?[\s\*]([A-Za-z_]\w*)\s*\(",
                       text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "for", "while", "return")))


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_c_header_symbols_exported():
    names = declared_functions("mlmq_b200.h")
    assert "sssp_init" in names and "mlmq_solver_create" in names
    syms = exported_symbols()
    missing = [n for n in names if n not in syms]
    assert not missing, missing
    for n in names:
        getattr(_lib.lib, n)  # resolvable through ctypes


def test_cxx_dropin_symbols_exported():
    """The reference's C++-linkage names (SS/SSSP/main.cu:15-17)."""
    syms = exported_symbols()
    for mangled in ("_Z9sssp_initiiPiS_S_", "_Z12sssp_re_initv",
                    "_Z17sssp_run_adaptivei10graph_info", "_Z12sssp_cp_dataPPi"):
        assert mangled in syms, mangled
    assert set(declared_functions("sssp_drop_in.h")) >= {
        "sssp_init", "sssp_re_init", "sssp_run_adaptive", "sssp_cp_data"}


def test_struct_layouts():
    assert ctypes.sizeof(_lib.GraphInfo) == 2 * 4 + 7 * 4
    assert ctypes.sizeof(_lib.Config) == 21 * 4


def test_config_defaults_are_the_reference_defaults(monkeypatch):
    for k in ("BENCH_DELTA", "BENCH_QUEUE", "MLMQ_WORK_BLOCKS"):
        monkeypatch.delenv(k, raising=False)
    c = mlmq.default_config()
    assert (c.queue_type, c.delta, c.l2_batch, c.bucket_num, c.bucket_max, c.min_read,
            c.large_degree, c.warps_per_block) == (19, 200000, 8, 16, 4, 8, 16, 16)


def test_config_environment(monkeypatch):
    monkeypatch.setenv("BENCH_DELTA", "1234")
    monkeypatch.setenv("MLMQ_WORK_BLOCKS", "7")
    monkeypatch.setenv("BENCH_QUEUE", "L1V_L2DQ")
    c = mlmq.default_config()
    assert (c.delta, c.work_blocks, c.queue_type) == (1234, 7, mlmq.MLMQ_L1V_L2DQ)
    monkeypatch.setenv("BENCH_QUEUE", "L1V_L2PQ")
    with pytest.raises(mlmq.MlmqError):
        mlmq.default_config()
    monkeypatch.setenv("BENCH_QUEUE", "L1SLF_L2DQ")
    monkeypatch.setenv("BENCH_DELTA", "0")
    with pytest.raises(mlmq.MlmqError):
        mlmq.default_config()


def test_errors_without_device_state():
    """Calls out of order fail with codes, never crash or exit."""
    assert _lib.lib.sssp_re_init() == _lib.MLMQ_ERR_STATE
    p = _lib.P_int()
    assert _lib.lib.sssp_cp_data(ctypes.byref(p)) == _lib.MLMQ_ERR_STATE
    assert _lib.lib.mlmq_solver_launch(None, 0, None) == _lib.MLMQ_ERR_ARG
    assert _lib.lib.mlmq_strerror(-4).decode().startswith("queue ring")
    # sources are checked before anything touches the device
    import numpy as np
    row = np.array([0, 1, 1], np.int32)
    col = np.array([1], np.int32)
    w = np.array([5], np.int32)
    out = np.empty((2, 2), np.int32)
    srcs = np.array([0, 2], np.int32)
    assert _lib.lib.mlmq_solve_host(2, 1, row.ctypes.data, col.ctypes.data, w.ctypes.data, 2,
                                    srcs.ctypes.data, out.ctypes.data, None) == _lib.MLMQ_ERR_ARG
    # no device memory has been pooled yet: releasing the cache is a no-op
    assert _lib.lib.mlmq_release_cached() == 0
    assert _lib.lib.mlmq_graph_prepare_light(None, 100) == _lib.MLMQ_ERR_ARG
    n = ctypes.c_int()
    assert _lib.lib.mlmq_server_poll_timed(None, None, None, None, 0,
                                           ctypes.byref(n)) == _lib.MLMQ_ERR_ARG
