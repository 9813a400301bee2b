"""The solve that allocates nothing (mlmq_sssp_solve_noalloc).

This entry point exists for callers that may not allocate device memory
while they run: code inside a framework that owns the device memory through
its own pool, processes that reserved all device memory at start-up, and
latency-critical paths where an allocation could block or fail.  It keeps
its queue workspace in a fixed array inside the library and reads the
caller's CSR in place, so the caller only provides the graph and the output
array.

The test calls it through the C ABI twice in a row and compares each result
with the allocating solver's on the same graph and source and with the CPU
oracle (exact equality: the distances are integers).  A call that ends early
(a 1 ms device time limit) leaves records in the shared workspace; the next
call must clear them and be exact again.  The file is named so that pytest
collects it last; it passes alone in a fresh process and after the other
tests.
"""
import ctypes

import numpy as np
import pytest

import oracle_lib
from mlmq_tpds_withl3_b200 import DeviceGraph, HostGraph, Solver, default_config
from mlmq_tpds_withl3_b200._lib import (MLMQ_ERR_QUEUE_FULL, MLMQ_ERR_RANGE, MLMQ_ERR_TIMEOUT,
                                        NOALLOC_MAX_ARCS, lib)

pytestmark = pytest.mark.gpu


def _device_csr(torch, g):
    return (torch.from_numpy(g.row.copy()).cuda(), torch.from_numpy(g.col.copy()).cuda(),
            torch.from_numpy(g.w.copy()).cuda())


def _noalloc(g, row, col, w, src, out, cfg):
    return lib.mlmq_sssp_solve_noalloc(g.n, g.m, row.data_ptr(), col.data_ptr(),
                                       w.data_ptr(), src, out.data_ptr(), ctypes.byref(cfg),
                                       None)


def test_noalloc_matches_allocating_solver_twice():
    import torch
    torch.cuda.init()
    g = HostGraph.grid(512, 512, drop_p=0.10, wmin=1000, wmax=100000, seed=1)
    assert g.m <= NOALLOC_MAX_ARCS
    row, col, w = _device_csr(torch, g)
    cfg = default_config(delta=200000)
    solver = Solver(DeviceGraph.upload(g), cfg)
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    for src in (0, 131072 + 256):  # two calls in a row on the shared workspace
        out.fill_(-1)
        torch.cuda.synchronize()
        rc = _noalloc(g, row, col, w, src, out, cfg)
        assert rc == 0, rc
        got = out.cpu().numpy()
        expected = solver.solve(src).dist()
        assert np.array_equal(got, expected), src
        ref, _ = oracle_lib.sssp_i32(g, src)
        assert np.array_equal(got, ref), src
    solver.close()


def test_noalloc_recovers_after_a_solve_that_ended_early():
    """A 1 ms device time limit on a solve that needs longer ends it with
    MLMQ_ERR_TIMEOUT and leaves records in the shared workspace; the next
    call clears the workspace first and returns exactly the allocating
    solver's distances."""
    import torch
    torch.cuda.init()
    g = HostGraph.grid(512, 512, drop_p=0.10, wmin=1000, wmax=100000, seed=1)
    row, col, w = _device_csr(torch, g)
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    rc = _noalloc(g, row, col, w, 0, out, default_config(delta=1000, timeout_ms=1))
    # ended early: the time limit, or a ring wait that the time limit cut short
    assert rc in (MLMQ_ERR_TIMEOUT, MLMQ_ERR_QUEUE_FULL), rc
    cfg = default_config(delta=200000)
    solver = Solver(DeviceGraph.upload(g), cfg)
    for src in (7, 200000):
        out.fill_(-1)
        torch.cuda.synchronize()
        assert _noalloc(g, row, col, w, src, out, cfg) == 0
        assert np.array_equal(out.cpu().numpy(), solver.solve(src).dist()), src
    solver.close()


def test_noalloc_rejects_graph_beyond_workspace():
    """A graph larger than the fixed workspace supports is refused up front
    (no kernel runs, so the arrays may be placeholders)."""
    import torch
    g = HostGraph.grid(1100, 1000, seed=3)
    assert g.m > NOALLOC_MAX_ARCS
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    cfg = default_config()
    rc = lib.mlmq_sssp_solve_noalloc(g.n, g.m, dummy.data_ptr(), dummy.data_ptr(),
                                     dummy.data_ptr(), 0, dummy.data_ptr(), ctypes.byref(cfg),
                                     None)
    assert rc == MLMQ_ERR_RANGE
