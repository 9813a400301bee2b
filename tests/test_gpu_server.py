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
        if i % 5 == 0:
            ref, _ = oracle_lib.sssp_i32(hgs[gi], src)
            assert np.array_equal(r["dist"], ref), (i, gi, src)
    s = summarize(recs)
    assert s["errors"] == 0 and s["queries"] == 80


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
