"""Host side of the served form on the CPU: the Poisson schedule, admission
(slot classes, result buffers, arrival order), completion bookkeeping and
the summary, against a fake server that completes queries after a few polls.
"""
import numpy as np
import pytest

from mlmq_tpds_withl3_b200.server import poisson_schedule, serve_poisson, summarize


class FakeKnobs:
    def __init__(self, work_blocks):
        self.work_blocks = work_blocks


class FakeGraph:
    def __init__(self, n):
        self.n = n


class FakeServer:
    """Slots of given CTA counts; a query finishes `polls` polls after it was
    submitted and writes its source into its result buffer."""

    def __init__(self, layout, polls=3, status_of=None):
        self.layout = list(layout)
        self.slots = len(layout)
        self.busy = [None] * self.slots
        self.polls = polls
        self.status_of = status_of or (lambda src: 0)
        self.next = 1
        self.submitted = []
        self.max_busy = 0

    def submit(self, dgraph, src, out, knobs=None):
        want = knobs.work_blocks if knobs is not None else 0
        free = [s for s in range(self.slots) if self.busy[s] is None and self.layout[s] >= want]
        if not free:
            return None
        s = min(free, key=lambda x: self.layout[x])
        tk = self.next
        self.next += 1
        out[:dgraph.n] = src
        self.busy[s] = [tk, self.polls, src]
        self.submitted.append((tk, src, s))
        self.max_busy = max(self.max_busy, sum(b is not None for b in self.busy))
        return tk

    def poll_timed(self):
        done = []
        for s, b in enumerate(self.busy):
            if b is None:
                continue
            b[1] -= 1
            if b[1] <= 0:
                done.append((b[0], self.status_of(b[2]), 0.5))
                self.busy[s] = None
        return done


class ListPool:
    def __init__(self, count, size):
        self.free = [np.zeros(size, np.int32) for _ in range(count)]

    def get(self):
        return self.free.pop() if self.free else None

    def put(self, buf):
        self.free.append(buf)


def test_poisson_schedule_is_seeded_and_ordered():
    a = poisson_schedule(1000.0, 500, [10, 20, 30], seed=4)
    b = poisson_schedule(1000.0, 500, [10, 20, 30], seed=4)
    assert a == b and len(a) == 500
    t = np.array([x[0] for x in a])
    assert np.all(np.diff(t) > 0)
    assert 0.3 < t[-1] < 0.7  # 500 arrivals at 1000/s
    assert all(0 <= src < [10, 20, 30][gi] for _, gi, src in a)


def test_every_query_served_once_with_its_own_result():
    graphs = [FakeGraph(8), FakeGraph(16)]
    sched = [(0.0, i % 2, i % 8) for i in range(60)]
    sv = FakeServer([2, 2, 2, 2], polls=2)
    recs = serve_poisson(sv, graphs, sched, keep=lambda i: True, pool=ListPool(4, 16),
                         timeout_s=10)
    assert len(recs) == 60 and all(r is not None for r in recs)
    assert sorted(src for _, src, _ in sv.submitted) == sorted(i % 8 for i in range(60))
    for i, r in enumerate(recs):
        assert r["graph"] == i % 2 and r["src"] == i % 8 and r["status"] == 0
        assert np.all(r["dist"] == i % 8) and len(r["dist"]) == graphs[i % 2].n
        assert r["solve_ms"] == 0.5 and r["finish"] >= r["start"] >= r["arrival"]
    assert sv.max_busy <= 4


def test_result_buffers_bound_the_queries_in_flight():
    graphs = [FakeGraph(4)]
    sched = [(0.0, 0, 1)] * 40
    sv = FakeServer([1] * 16, polls=3)
    serve_poisson(sv, graphs, sched, pool=ListPool(3, 4), timeout_s=10)
    assert sv.max_busy == 3


def test_a_full_slot_class_does_not_hold_back_other_queries():
    """Graph 0 needs a wide slot (work_blocks 8); with the one wide slot busy
    the small-slot queries behind it are still admitted in arrival order."""
    graphs = [FakeGraph(4), FakeGraph(4)]
    knobs = [FakeKnobs(8), FakeKnobs(0)]
    sched = [(0.0, 0, 0), (0.0, 0, 1)] + [(0.0, 1, 2)] * 6
    sv = FakeServer([8, 1, 1, 1], polls=50)
    serve_poisson(sv, graphs, sched, pool=ListPool(8, 4), timeout_s=10, knobs=knobs)
    order = [src for _, src, _ in sv.submitted]
    # the second wide query waited for the wide slot; small ones went first
    assert order[0] == 0 and order.index(1) > order.index(2)
    wide = [slot for _, src, slot in sv.submitted if src in (0, 1)]
    assert wide == [0, 0]


def test_summary_counts_errors_per_graph():
    graphs = [FakeGraph(4), FakeGraph(4)]
    sched = [(0.0, i % 2, i) for i in range(20)]
    sv = FakeServer([1, 1], polls=1, status_of=lambda src: -3 if src % 5 == 0 else 0)
    recs = serve_poisson(sv, graphs, sched, pool=ListPool(2, 4), timeout_s=10)
    s = summarize(recs, ["a", "b"])
    assert s["queries"] == 20 and s["errors"] == 4 and s["error_codes"] == {"-3": 4}
    # sources 0 and 10 ran on graph a, 5 and 15 on graph b
    assert s["per_graph"]["a"]["queries"] == 10 and s["per_graph"]["a"]["errors"] == 2
    assert s["per_graph"]["b"]["errors"] == 2
    assert s["p99_ms"] >= s["p50_ms"] >= 0 and s["qps"] > 0
    assert s["per_graph"]["a"]["solve_ms_mean"] == pytest.approx(0.5)


def test_serving_gives_up_after_its_time_limit_with_statuses():
    """A query that never completes ends the run at the host time limit;
    every query gets a record: the one in flight and the one still waiting
    carry HOST_TIMEOUT, and the summary counts them as errors."""
    from mlmq_tpds_withl3_b200.server import HOST_TIMEOUT
    graphs = [FakeGraph(4)]
    sv = FakeServer([1], polls=10**9)
    recs = serve_poisson(sv, graphs, [(0.0, 0, 1), (0.0, 0, 2)], pool=ListPool(2, 4),
                         timeout_s=0.2)
    assert [r["status"] for r in recs] == [HOST_TIMEOUT, HOST_TIMEOUT]
    assert recs[0]["start"] is not None and recs[1]["start"] is None
    s = summarize(recs)
    assert s["finished"] == 0 and s["errors"] == 2 and s["qps"] == 0.0


def test_serving_reports_finished_and_timed_out_queries_together():
    graphs = [FakeGraph(4)]

    class Stuck(FakeServer):
        def poll_timed(self):
            done = super().poll_timed()
            return [d for d in done if d[0] != 2]  # ticket 2 never completes

    sv = Stuck([1, 1], polls=1)
    from mlmq_tpds_withl3_b200.server import HOST_TIMEOUT
    recs = serve_poisson(sv, graphs, [(0.0, 0, k) for k in range(3)], pool=ListPool(3, 4),
                         timeout_s=0.3)
    statuses = sorted(str(r["status"]) for r in recs)
    assert statuses == ["0", "0", HOST_TIMEOUT]
    s = summarize(recs)
    assert s["finished"] == 2 and s["errors"] == 1 and s["error_codes"] == {HOST_TIMEOUT: 1}
