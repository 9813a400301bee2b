"""Continuous-batching server: queries on graphs of different sizes arrive
while others run; every result equals the oracle and the same query solved
alone."""
import numpy as np
import pytest

import oracle_lib
from mlmq_tpds_withl3_b200 import DeviceGraph, HostGraph, Solver
from mlmq_tpds_withl3_b200.server import Server, poisson_schedule, serve_poisson, summarize

pytestmark = pytest.mark.gpu


def _graphs():
    return [HostGraph.grid(128, 128, seed=41), HostGraph.grid(300, 260, seed=42),
            HostGraph.knn(30000, seed=43), HostGraph.rmat(13, seed=44)]


def test_served_results_equal_oracle_and_alone():
    hgs = _graphs()
    dgs = [DeviceGraph.upload(g) for g in hgs]
    sv = Server(slots=12, max_vertices=max(dg.slots for dg in dgs), lifetime_s=120)
    sched = poisson_schedule(rate=3000.0, count=80, graphs_n=[g.n for g in hgs], seed=7)
    recs = serve_poisson(sv, dgs, sched, keep=lambda i: True, timeout_s=60)
    sv.close()
    assert all(r["status"] == 0 for r in recs)
    # device solve time: positive and inside the host-seen submit-to-result span
    assert all(0 < r["solve_ms"] <= (r["finish"] - r["start"]) * 1e3 + 1.0 for r in recs)
    # queries overlapped on the device: some started before others finished
    overlap = sum(1 for a, b in zip(recs, recs[1:]) if b["start"] < a["finish"])
    assert overlap > 0
    alone = [Solver(dg) for dg in dgs]
    for i, r in enumerate(recs):
        gi, src = r["graph"], r["src"]
        solo = alone[gi].solve(src).dist()
        assert np.array_equal(r["dist"], solo), (i, gi, src)
        # every served result against the oracle (SS/SSSP/sssp_run.cu:849-859
        # checks every solve the same way)
        ref, _ = oracle_lib.sssp_i32(hgs[gi], src)
        assert np.array_equal(r["dist"], ref), (i, gi, src)
        # the device-computed digest of the same result
        assert r["digest"] == oracle_lib.digest(ref), (i, gi, src)
    s = summarize(recs)
    assert s["errors"] == 0 and s["queries"] == 80 and s["finished"] == 80


def test_per_query_settings_give_the_same_result():
    """Queries submitted with their own delta / topup / run-ahead bound /
    read window return the same distances as the oracle."""
    from mlmq_tpds_withl3_b200 import default_config
    g = HostGraph.grid(200, 180, seed=46)
    dg = DeviceGraph.upload(g)
    sv = Server(slots=4, max_vertices=g.n, lifetime_s=60)
    import torch
    knobs = [default_config(delta=5000, topup=32, l1_ahead=1, bucket_max=2),
             default_config(delta=400000, topup=0, l1_ahead=0, bucket_max=8), None]
    bufs = [torch.empty(g.n, dtype=torch.int32, pin_memory=True) for _ in knobs]
    tks = [sv.submit(dg, 9, b, k) for b, k in zip(bufs, knobs)]
    assert all(t is not None for t in tks)
    done = {}
    import time
    t0 = time.time()
    while len(done) < len(tks) and time.time() - t0 < 30:
        for tk, st in sv.poll():
            done[tk] = st
    sv.close()
    assert all(done.get(t) == 0 for t in tks)
    ref, _ = oracle_lib.sssp_i32(g, 9)
    for b in bufs:
        assert np.array_equal(b.numpy(), ref)


def test_light_heavy_queries_need_prepared_counts():
    """A running server holds every SM, so light/heavy queries need their
    light-arc counts prepared before it starts; unprepared ones are refused
    at once (no device work inside submit), prepared ones are exact."""
    from mlmq_tpds_withl3_b200 import MlmqError, default_config
    from mlmq_tpds_withl3_b200._lib import MLMQ_ERR_STATE
    import torch
    import time
    g = HostGraph.rmat(13, seed=48)
    dg = DeviceGraph.upload(g)
    dg.prepare_light(20000)
    sv = Server(slots=3, max_vertices=dg.slots + dg.n, lifetime_s=60)
    buf = torch.empty(g.n, dtype=torch.int32, pin_memory=True)
    with pytest.raises(MlmqError) as ei:
        sv.submit(dg, 0, buf, default_config(light_heavy=1, delta=30000))
    assert ei.value.code == MLMQ_ERR_STATE
    del ei
    tk = sv.submit(dg, 0, buf, default_config(light_heavy=1, bucket_sync=1, delta=20000))
    done = {}
    t0 = time.time()
    while tk not in done and time.time() - t0 < 30:
        for t, st in sv.poll():
            done[t] = st
    sv.close()
    assert done.get(tk) == 0
    ref, _ = oracle_lib.sssp_i32(g, 0)
    assert np.array_equal(buf.numpy(), ref)


def test_slot_layout_and_slot_choice():
    """Slots of different sizes: a query asking for 6 CTAs gets the wide slot
    and waits while it is taken; results stay exact."""
    from mlmq_tpds_withl3_b200 import default_config
    import torch
    import time
    g = HostGraph.grid(150, 150, seed=47)
    dg = DeviceGraph.upload(g)
    sv = Server(slots=0, max_vertices=dg.slots, layout=[1, 2, 6], lifetime_s=60)
    assert sv.layout == [1, 2, 6] and sv.grid == 9
    wide = default_config(work_blocks=6)
    bufs = [torch.empty(g.n, dtype=torch.int32, pin_memory=True) for _ in range(4)]
    t_wide = sv.submit(dg, 3, bufs[0], wide)
    assert t_wide is not None
    assert sv.submit(dg, 4, bufs[1], wide) is None  # the only wide slot is taken
    t_a = sv.submit(dg, 5, bufs[2])                 # smallest free slot
    t_b = sv.submit(dg, 6, bufs[3])
    assert t_a is not None and t_b is not None
    done = {}
    t0 = time.time()
    while len(done) < 3 and time.time() - t0 < 30:
        for tk, st in sv.poll():
            done[tk] = st
    sv.close()
    assert done == {t_wide: 0, t_a: 0, t_b: 0}
    for src, b in ((3, bufs[0]), (5, bufs[2]), (6, bufs[3])):
        ref, _ = oracle_lib.sssp_i32(g, src)
        assert np.array_equal(b.numpy(), ref), src


def test_server_busy_and_stop():
    g = HostGraph.grid(64, 64, seed=45)
    dg = DeviceGraph.upload(g)
    import torch
    sv = Server(slots=2, max_vertices=g.n, lifetime_s=60)
    bufs = [torch.empty(g.n, dtype=torch.int32, pin_memory=True) for _ in range(3)]
    t1 = sv.submit(dg, 0, bufs[0])
    t2 = sv.submit(dg, 1, bufs[1])
    assert t1 is not None and t2 is not None
    assert sv.submit(dg, 2, bufs[2]) is None  # both slots busy
    done = {}
    import time
    t0 = time.time()
    while len(done) < 2 and time.time() - t0 < 30:
        for tk, st in sv.poll():
            done[tk] = st
    assert done == {t1: 0, t2: 0}
    ref0, _ = oracle_lib.sssp_i32(g, 0)
    assert np.array_equal(bufs[0].numpy(), ref0)
    sv.close()


def test_queries_after_the_server_kernel_ended_are_reported():
    """A server whose lifetime has run out takes no queries: a submit before
    the host noticed is reported by poll as MLMQ_ERR_STATE (no result was
    written), and submits after that fail at once."""
    import time
    import torch
    from mlmq_tpds_withl3_b200 import MlmqError
    from mlmq_tpds_withl3_b200._lib import MLMQ_ERR_STATE
    g = HostGraph.grid(64, 64, seed=49)
    dg = DeviceGraph.upload(g)
    sv = Server(slots=2, max_vertices=g.n, lifetime_s=1.0)
    buf = torch.empty(g.n, dtype=torch.int32, pin_memory=True)
    t0 = sv.submit(dg, 0, buf)
    done = {}
    t = time.time()
    while t0 not in done and time.time() - t < 10:
        done.update(dict(sv.poll()))
    assert done.get(t0) == 0
    time.sleep(2.0)  # the server kernel's lifetime ends while it is idle
    late = sv.submit(dg, 1, buf)
    res = {}
    t = time.time()
    while late not in res and time.time() - t < 10:
        res.update(dict(sv.poll()))
    assert res.get(late) == MLMQ_ERR_STATE
    with pytest.raises(MlmqError) as ei:
        sv.submit(dg, 2, buf)
    assert ei.value.code == MLMQ_ERR_STATE
    del ei
    sv.close()


def test_slot_whose_ctas_cannot_meet_reports_and_retires(monkeypatch):
    """Bounded slot barrier: with one CTA of slot 0 made to leave the kernel
    after its first solve (a CTA that never arrives, as a flag that nothing
    sets), the slot's other CTAs wait for it only until the query's own time
    limit plus the meeting margin, then report the query as MLMQ_ERR_TIMEOUT
    and retire the slot; queries keep running, exact, on the other slots."""
    import time
    import torch
    from mlmq_tpds_withl3_b200 import default_config
    from mlmq_tpds_withl3_b200._lib import MLMQ_ERR_TIMEOUT
    g = HostGraph.grid(96, 96, seed=50)
    dg = DeviceGraph.upload(g)
    monkeypatch.setenv("MLMQ_SERVER_TEST_ABSENT_CTA", "1")
    monkeypatch.setenv("MLMQ_SERVER_MEET_MS", "300")
    sv = Server(slots=0, max_vertices=g.n, layout=[2, 2],
                cfg=default_config(warps_per_block=8, timeout_ms=500), lifetime_s=60)
    bufs = [torch.empty(g.n, dtype=torch.int32, pin_memory=True) for _ in range(4)]
    first = [sv.submit(dg, s, bufs[s]) for s in (0, 1)]
    done = {}
    t = time.time()
    while len(done) < 2 and time.time() - t < 20:
        done.update(dict(sv.poll()))
    elapsed = time.time() - t
    assert sorted(done.values()) == [MLMQ_ERR_TIMEOUT, 0], done
    assert elapsed < 10
    busy, running = sv.busy()
    assert busy == 1 and running  # the lost slot stays out of service
    ok_slot_buf = [bufs[s] for s, tk in zip((0, 1), first) if done[tk] == 0][0]
    ref0 = [oracle_lib.sssp_i32(g, s)[0] for s in (0, 1)]
    assert any(np.array_equal(ok_slot_buf.numpy(), r) for r in ref0)
    # later queries go to the remaining slot and stay exact
    for src in (5, 6):
        tk = sv.submit(dg, src, bufs[2])
        assert tk is not None
        res = {}
        t = time.time()
        while tk not in res and time.time() - t < 10:
            res.update(dict(sv.poll()))
        assert res.get(tk) == 0
        assert np.array_equal(bufs[2].numpy(), oracle_lib.sssp_i32(g, src)[0])
    sv.close()


def test_freeing_while_a_server_runs_does_not_wait_for_it():
    """Solvers, batches and graphs dropped while a server kernel runs go back
    to the pools without waiting for that kernel (cudaFree would synchronise
    the device, i.e. wait for the server's whole lifetime); a graph whose
    handle is closed while a served query still reads it stays allocated
    until that query has reported, and the result is exact."""
    import time
    import torch
    from mlmq_tpds_withl3_b200 import BatchSolver
    g = HostGraph.grid(128, 128, seed=51)
    dg1 = DeviceGraph.upload(g)
    s1 = Solver(dg1)
    s1.solve(3)
    b1 = BatchSolver(2, dg1.slots)
    b1.run([(dg1, 1), (dg1, 2)])
    dg2 = DeviceGraph.upload(g)
    sv = Server(slots=2, max_vertices=dg1.slots, lifetime_s=60)
    t0 = time.time()
    s1.close()
    b1.close()
    dg1.close()
    assert time.time() - t0 < 5.0
    buf = torch.empty(g.n, dtype=torch.int32, pin_memory=True)
    tk = sv.submit(dg2, 17, buf)
    dg2.close()  # the server's reference keeps the graph until the query reports
    done = {}
    t = time.time()
    while tk not in done and time.time() - t < 20:
        done.update(dict(sv.poll()))
    assert done.get(tk) == 0
    sv.close()
    assert np.array_equal(buf.numpy(), oracle_lib.sssp_i32(g, 17)[0])


def test_server_with_wide_tiles_needs_them_prepared():
    """A server reading 64-byte tiles refuses a graph whose wide tiles were
    not built before it started (nothing is built inside submit); prepared
    graphs give exact results."""
    import time
    import torch
    from mlmq_tpds_withl3_b200 import MlmqError, default_config
    from mlmq_tpds_withl3_b200._lib import MLMQ_ERR_STATE
    g = HostGraph.knn(20000, seed=52)
    a, b = DeviceGraph.upload(g), DeviceGraph.upload(g)
    a.prepare_tiles(2)
    sv = Server(slots=2, max_vertices=g.n, cfg=default_config(warps_per_block=8, vertex_tiles=2),
                lifetime_s=60)
    buf = torch.empty(g.n, dtype=torch.int32, pin_memory=True)
    with pytest.raises(MlmqError) as ei:
        sv.submit(b, 0, buf)
    assert ei.value.code == MLMQ_ERR_STATE
    del ei
    tk = sv.submit(a, 11, buf)
    done = {}
    t = time.time()
    while tk not in done and time.time() - t < 20:
        done.update(dict(sv.poll()))
    sv.close()
    assert done.get(tk) == 0
    assert np.array_equal(buf.numpy(), oracle_lib.sssp_i32(g, 11)[0])
