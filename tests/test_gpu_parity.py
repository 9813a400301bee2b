"""Bit-exact parity of the sm_100a solver with the oracle (GPU tests).

Every comparison is exact int32 equality, INT_MAX for unreachable vertices:
shortest-path distances with non-negative integer weights are unique."""
import json
import os

import numpy as np
import pytest

import oracle_lib
from fixtures import golden_graphs
from mlmq_tpds_withl3_b200 import (DeviceGraph, HostGraph, Solver, default_config,
                                   MLMQ_L1V_L2DQ)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
pytestmark = pytest.mark.gpu


def _manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def _golden_cases():
    for name, entry in sorted(_manifest().items()):
        for src in sorted(entry["sources"], key=int):
            yield name, int(src)


@pytest.mark.parametrize("name,src", list(_golden_cases()))
def test_golden_fixtures(name, src):
    entry = _manifest()[name]
    g = HostGraph.read_gr(os.path.join(GOLDEN, entry["file"]))
    gold = np.fromfile(os.path.join(GOLDEN, entry["sources"][str(src)]["file"]), dtype=np.int32)
    s = Solver(DeviceGraph.upload(g))
    assert np.array_equal(s.solve(src).dist(), gold)


def test_source_switching_reuses_workspace():
    """Sources 0, 1030, 2050, 0 on one solver, as the reference's reset check
    (scripts/multigpu/run_supplement_checks.py:44-54)."""
    g, _ = golden_graphs()["supplement2052"]
    s = Solver(DeviceGraph.upload(g))
    for src in (0, 1030, 2050, 0):
        ref, _ = oracle_lib.sssp_i32(g, src)
        assert np.array_equal(s.solve(src).dist(), ref), src


def test_c1_grid512_bit_exact():
    """Config 1 at full size: 512x512 grid, 10% edges dropped, w U{1000..100000},
    source 0, delta 200000, L1SLF_L2DQ."""
    g = HostGraph.grid(512, 512, drop_p=0.10, wmin=1000, wmax=100000, seed=1)
    ref, work = oracle_lib.sssp_i32(g, 0)
    s = Solver(DeviceGraph.upload(g), {"delta": 200000})
    for _ in range(3):
        assert np.array_equal(s.solve(0).dist(), ref)
    st = s.stats()
    assert st["relaxed"] >= work  # every settled vertex scanned at least once


@pytest.mark.parametrize("cfg", [
    {"bucket_max": 1, "l2_batch": 1, "min_read": 1},
    {"bucket_num": 4, "bucket_max": 4, "delta": 20000},
    {"bucket_num": 31, "bucket_max": 8, "l2_batch": 4},
    {"delta": 1},
    {"delta": 1 << 30},
    {"queue_type": MLMQ_L1V_L2DQ},
    {"warps_per_block": 4, "work_blocks": 3},
    {"large_degree": 1},
    {"l1_spill": 1},
    {"l2_cap_log2": 18, "l3_cap_log2": 18},
    {"l1_keep": 8},
    {"l1_keep": 32, "queue_type": MLMQ_L1V_L2DQ},
    {"relax_precheck": 0},
    {"relax_unroll": 1},
    {"relax_unroll": 2, "large_degree": 4},
    {"relax_unroll": 4, "relax_precheck": 0, "warps_per_block": 24},
    {"relax_unroll": 1, "warps_per_block": 31},
    {"vertex_tiles": 0},
    {"vertex_tiles": 0, "relax_precheck": 0, "relax_unroll": 1},
    {"vertex_tiles": 2},
    {"vertex_tiles": 2, "light_heavy": 1, "bucket_sync": 1, "delta": 30000},
    {"vertex_tiles": 2, "relax_unroll": 1, "large_degree": 4096},
    {"topup": 32},
    {"topup": 16, "l1_ahead": 0, "min_read": 1},
    {"l1_ahead": 1, "delta": 2000},
    {"bucket_sync": 1},
    {"bucket_sync": 1, "bucket_max": 1, "l1_ahead": 1, "delta": 3000},
    {"light_heavy": 1},
    {"light_heavy": 1, "bucket_sync": 1, "bucket_max": 1, "delta": 20000},
    {"light_heavy": 1, "delta": 1},
])
def test_queue_configurations(cfg):
    """Any queue configuration gives the same exact distances (ordering only
    changes the amount of work)."""
    g = HostGraph.grid(128, 96, seed=4)
    ref, _ = oracle_lib.sssp_i32(g, 5)
    s = Solver(DeviceGraph.upload(g), cfg)
    assert np.array_equal(s.solve(5).dist(), ref)


def test_live_solvers_with_different_cta_sizes():
    """A solver created after another one with a larger CTA must not break
    the first one's launches (the kernel's shared-memory limit is shared)."""
    g = HostGraph.grid(96, 96, seed=6)
    dg = DeviceGraph.upload(g)
    big = Solver(dg, {"warps_per_block": 24})
    small = Solver(dg, {"warps_per_block": 4})
    ref, _ = oracle_lib.sssp_i32(g, 7)
    for s in (big, small, big):
        assert np.array_equal(s.solve(7).dist(), ref)


def test_split_heavy_vertices_exact():
    """Vertices of more than 1024 arcs are relaxed as 512-arc pieces taken by
    different warps; single, batched and tile-less solves stay exact."""
    from mlmq_tpds_withl3_b200 import BatchSolver
    g = HostGraph.rmat(16, seed=13)
    dg = DeviceGraph.upload(g)
    assert dg.pieces > 0 and dg.slots == g.n + dg.pieces
    srcs = [0, 1, 2]
    ref, _ = oracle_lib.sssp_many(g, srcs)
    s = Solver(dg)
    flat = Solver(dg, {"vertex_tiles": 0})
    for k, src in enumerate(srcs):
        assert np.array_equal(s.solve(src).dist(), ref[k]), src
        assert np.array_equal(flat.solve(src).dist(), ref[k]), src
    b = BatchSolver(len(srcs), dg.slots, {"topup": 32})
    b.run([(dg, x) for x in srcs])
    for k in range(len(srcs)):
        assert np.array_equal(b.dist(k), ref[k])
    # narrow buckets push pieces through L3 as well
    t = Solver(dg, {"bucket_num": 2, "bucket_max": 1, "delta": 3000, "timeout_ms": 15000})
    assert np.array_equal(t.solve(0).dist(), ref[0])
    # wide tiles (8 inline arcs) with split vertices, single and batched
    wide = Solver(dg, {"vertex_tiles": 2})
    for k, src in enumerate(srcs):
        assert np.array_equal(wide.solve(src).dist(), ref[k]), src
    bw = BatchSolver(len(srcs), dg.slots, {"vertex_tiles": 2, "topup": 32})
    bw.run([(dg, x) for x in srcs])
    for k in range(len(srcs)):
        assert np.array_equal(bw.dist(k), ref[k])
    # light/heavy split (heavy arcs and heavy pieces one bucket later),
    # single and batched, also through narrow buckets and L3
    for cfg in ({"light_heavy": 1}, {"light_heavy": 1, "delta": 20000, "bucket_sync": 1,
                                     "bucket_max": 1}):
        lh = Solver(dg, cfg)
        for k, src in enumerate(srcs):
            assert np.array_equal(lh.solve(src).dist(), ref[k]), (cfg, src)
    t2 = Solver(dg, {"light_heavy": 1, "bucket_num": 2, "bucket_max": 1, "delta": 3000,
                     "timeout_ms": 15000})
    assert np.array_equal(t2.solve(1).dist(), ref[1])
    bd = BatchSolver(len(srcs), dg.slots + dg.n, {"light_heavy": 1, "topup": 16})
    bd.run([(dg, x) for x in srcs])
    for k in range(len(srcs)):
        assert np.array_equal(bd.dist(k), ref[k])


def test_graph_build_paths_and_pooled_memory():
    """Graphs built from host arrays and from device arrays find the same
    heavy vertices (found on the device) and solve exactly; graphs and
    solvers built and dropped over and over reuse pooled device memory, and
    releasing the pool's cache leaves live graphs and solvers intact."""
    import torch
    from mlmq_tpds_withl3_b200._lib import lib
    g = HostGraph.rmat(15, seed=21)
    ref, _ = oracle_lib.sssp_i32(g, 3)
    up = DeviceGraph.upload(g)
    row, col, w = (torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).cuda()
                   for a in (g.row, g.col, g.w))
    wrapped = DeviceGraph.wrap_device(g.n, g.m, row.data_ptr(), col.data_ptr(), w.data_ptr())
    assert up.pieces > 0 and wrapped.pieces == up.pieces
    live = Solver(wrapped)
    assert np.array_equal(live.solve(3).dist(), ref)
    for k in range(4):
        dg = DeviceGraph.upload(g)
        s = Solver(dg, {"light_heavy": k % 2})
        assert np.array_equal(s.solve(3).dist(), ref), k
        s.close()
        dg.close()
    assert lib.mlmq_release_cached() == 0
    assert np.array_equal(live.solve(3).dist(), ref)
    assert np.array_equal(Solver(up).solve(3).dist(), ref)


def test_host_buffer_call_many_sources():
    """mlmq_solve_host: upload, one solve per source (solving the next while
    copying the last out), distances row by row; pageable and pinned output,
    one source and none."""
    import ctypes
    import torch
    from mlmq_tpds_withl3_b200 import solve_host, default_config
    from mlmq_tpds_withl3_b200._lib import lib, check
    g = HostGraph.rmat(14, seed=31)
    srcs = [0, 7, 300, 7, 4095]
    ref, _ = oracle_lib.sssp_many(g, srcs)
    assert np.array_equal(solve_host(g, srcs), ref)
    assert np.array_equal(solve_host(g, srcs[2:3], {"light_heavy": 1}), ref[2:3])
    assert solve_host(g, []).shape == (0, g.n)
    out = torch.empty((len(srcs), g.n), dtype=torch.int32).pin_memory()
    sa = np.asarray(srcs, np.int32)
    check(lib.mlmq_solve_host(g.n, g.m, g.row.ctypes.data, g.col.ctypes.data, g.w.ctypes.data,
                              len(srcs), sa.ctypes.data, out.data_ptr(),
                              ctypes.byref(default_config(vertex_tiles=0))), "mlmq_solve_host")
    assert np.array_equal(out.numpy(), ref)


def test_knn_and_rmat_medium():
    for g in (HostGraph.knn(200000, seed=2), HostGraph.rmat(16, seed=3)):
        s = Solver(DeviceGraph.upload(g))
        for src in (0, g.n // 2 + 1):
            ref, _ = oracle_lib.sssp_i32(g, src)
            assert np.array_equal(s.solve(src).dist(), ref), (g.name, src)


def test_l3_far_records_exact():
    """A two-bucket window of narrow buckets sends most records beyond the
    window to the L3 ring; results stay exact and L3 is exercised."""
    g = HostGraph.rmat(14, seed=8)
    ref, _ = oracle_lib.sssp_i32(g, 0)
    s = Solver(DeviceGraph.upload(g), {"l2_cap_log2": 18, "bucket_num": 2, "bucket_max": 1,
                                        "delta": 5000, "timeout_ms": 10000})
    assert np.array_equal(s.solve(0).dist(), ref)
    assert s.stats()["l3_pushed"] > 0


def test_l2_pressure_path_exact():
    """One bucket wide enough to hold every distance fills its ring past the
    pressure threshold, so later pushes divert to L3; results stay exact."""
    g = HostGraph.rmat(17, seed=9)
    ref, _ = oracle_lib.sssp_i32(g, 1)
    s = Solver(DeviceGraph.upload(g), {"l2_cap_log2": 18, "bucket_num": 1, "bucket_max": 1,
                                        "delta": 1 << 30, "l1_spill": 1,
                                        "timeout_ms": 10000})
    assert np.array_equal(s.solve(1).dist(), ref)


def test_l3_one_record_per_vertex_bounds_the_ring():
    """Narrow buckets over a two-bucket window send most pushes of an R-MAT
    graph to L3, whose ring (2^19 slots) is smaller than the pushes it sees:
    L3 keeps one record per vertex (n = 2^18), so the ring never fills and
    the result stays exact."""
    g = HostGraph.rmat(18, seed=12)
    ref, _ = oracle_lib.sssp_i32(g, 0)
    s = Solver(DeviceGraph.upload(g), {"bucket_num": 2, "bucket_max": 1, "delta": 2000,
                                        "l3_cap_log2": 19, "timeout_ms": 15000})
    assert np.array_equal(s.solve(0).dist(), ref)
    assert s.stats()["l3_pushed"] > 0


def test_full_l3_ring_is_reported_not_asserted():
    """Capacity: narrow buckets send almost every record of a 1M-vertex
    R-MAT graph beyond the window, more distinct vertices than a 2^18-slot
    L3 ring holds.  A push that finds the ring full waits (bounded) and the
    solve ends with MLMQ_ERR_QUEUE_FULL -- a status, never a device assert --
    and the next solve with a fitting ring is exact."""
    from mlmq_tpds_withl3_b200 import MlmqError
    from mlmq_tpds_withl3_b200._lib import MLMQ_ERR_QUEUE_FULL, MLMQ_ERR_TIMEOUT
    g = HostGraph.rmat(20, seed=15)
    dg = DeviceGraph.upload(g)
    tight = Solver(dg, {"bucket_num": 2, "bucket_max": 1, "delta": 2000,
                        "l3_cap_log2": 18, "timeout_ms": 2000})
    ref, _ = oracle_lib.sssp_i32(g, 0)
    try:
        got = tight.solve(0).dist()
    except MlmqError as e:  # the expected outcome: the ring filled
        assert e.code in (MLMQ_ERR_QUEUE_FULL, MLMQ_ERR_TIMEOUT)
    else:  # had every record fitted after all, the result must be exact
        assert np.array_equal(got, ref)
    tight.close()
    after = Solver(dg)
    assert np.array_equal(after.solve(0).dist(), ref)
    after.close()
    dg.close()


def test_transformed_graphs_solve_exact():
    """G+ (chain shortcuts) and the BFS-reordered graph on the GPU: the same
    distances as the original graph, permuted for the reordering."""
    g = HostGraph.grid(256, 256, drop_p=0.25, seed=31)
    src = 123
    ref, _ = oracle_lib.sssp_i32(g, src)
    gp, st = g.chain_shortcuts(source=src)
    assert st["shortcuts"] > 0
    assert np.array_equal(Solver(DeviceGraph.upload(gp)).solve(src).dist(), ref)
    r, perm, inv = g.reorder_bfs(src)
    got = Solver(DeviceGraph.upload(r)).solve(int(inv[src])).dist()
    assert np.array_equal(got[inv], ref)


def test_timeout_is_reported_not_hung():
    """A 1 ms device time limit on a graph that needs longer ends the solve
    with MLMQ_ERR_TIMEOUT; the next solve with a normal limit is exact."""
    from mlmq_tpds_withl3_b200 import MlmqError
    from mlmq_tpds_withl3_b200._lib import MLMQ_ERR_TIMEOUT
    g = HostGraph.grid(512, 512, seed=1)
    dg = DeviceGraph.upload(g)
    s = Solver(dg, {"timeout_ms": 1, "delta": 1000})
    with pytest.raises(MlmqError) as ei:
        s.solve(0)
    assert ei.value.code == MLMQ_ERR_TIMEOUT
    del ei  # its traceback would keep this frame's solvers alive until a GC pass
    s.close()
    ref, _ = oracle_lib.sssp_i32(g, 0)
    after = Solver(dg)
    assert np.array_equal(after.solve(0).dist(), ref)
    after.close()
    dg.close()


def test_dropin_entry_points_with_device_csr():
    """sssp_init / sssp_re_init / sssp_run_adaptive / sssp_cp_data on a
    caller-owned device CSR, as SS/SSSP/main.cu:204-215 calls them."""
    import torch
    from mlmq_tpds_withl3_b200 import (sssp_cp_data, sssp_init, sssp_re_init,
                                       sssp_run_adaptive)
    g = HostGraph.grid(200, 150, seed=21)
    row = torch.from_numpy(g.row.copy()).cuda()
    col = torch.from_numpy(g.col.copy()).cuda()
    w = torch.from_numpy(g.w.copy()).cuda()
    os.environ["BENCH_WARMUPS"] = "0"
    os.environ["BENCH_REPEATS"] = "1"
    try:
        sssp_init(g.n, g.m, row.data_ptr(), col.data_ptr(), w.data_ptr())
        for src in (0, 777):
            sssp_re_init()
            sssp_run_adaptive(src, g.info())
            ref, _ = oracle_lib.sssp_i32(g, src)
            assert np.array_equal(sssp_cp_data(), ref)
    finally:
        del os.environ["BENCH_WARMUPS"], os.environ["BENCH_REPEATS"]
