"""Batched multi-source solving: every query of a launch is bit-exact against
the oracle, whatever mix of sources and graphs shares the launch."""
import numpy as np
import pytest

import oracle_lib
from fixtures import golden_graphs
from mlmq_tpds_withl3_b200 import BatchSolver, DeviceGraph, HostGraph

pytestmark = pytest.mark.gpu


def test_many_sources_one_graph():
    g = HostGraph.grid(256, 256, seed=31)
    dg = DeviceGraph.upload(g)
    rng = np.random.default_rng(5)
    srcs = [int(s) for s in rng.choice(g.n, 48, replace=False)]
    ref, _ = oracle_lib.sssp_many(g, srcs)
    b = BatchSolver(64, g.n)
    b.run([(dg, s) for s in srcs])
    for q, s in enumerate(srcs):
        assert np.array_equal(b.dist(q), ref[q]), (q, s)


def test_uneven_graphs_in_one_launch():
    graphs = [HostGraph.grid(100, 80, seed=2), HostGraph.knn(20000, seed=3),
              HostGraph.rmat(13, seed=4)]
    graphs += [g for g, _ in golden_graphs().values()]
    dgs = [DeviceGraph.upload(g) for g in graphs]
    queries, refs = [], []
    for g, dg in zip(graphs, dgs):
        for s in (0, g.n - 1):
            queries.append((dg, s))
            refs.append(oracle_lib.sssp_i32(g, s)[0])
    b = BatchSolver(len(queries), max(dg.slots for dg in dgs))
    b.run(queries)
    for q, ref in enumerate(refs):
        assert np.array_equal(b.dist(q), ref), q


def test_graph_replay_and_recapture():
    g = HostGraph.grid(192, 160, seed=7)
    dg = DeviceGraph.upload(g)
    b = BatchSolver(16, g.n)
    set1 = [0, 5, 999, 30000]
    set2 = [1, 2, 3, 4, 5, 6]
    for srcs in (set1, set1, set2, set1):
        b.run([(dg, s) for s in srcs], use_graph=True)
        ref, _ = oracle_lib.sssp_many(g, srcs)
        for q in range(len(srcs)):
            assert np.array_equal(b.dist(q), ref[q])


def test_batch_matches_plain_solver_on_larger_grid():
    """Size-independent property at a larger size: each batched query equals
    the single-source solver's result (itself checked against the oracle on
    two of the sources)."""
    from mlmq_tpds_withl3_b200 import Solver
    g = HostGraph.grid(1024, 1024, seed=9)
    dg = DeviceGraph.upload(g)
    rng = np.random.default_rng(11)
    srcs = [int(s) for s in rng.choice(g.n, 64, replace=False)]
    b = BatchSolver(64, g.n)
    b.run([(dg, s) for s in srcs], use_graph=True)
    plain = Solver(dg)
    for q, s in enumerate(srcs):
        assert np.array_equal(b.dist(q), plain.solve(s).dist()), q
    for q in (0, 63):
        ref, _ = oracle_lib.sssp_i32(g, srcs[q])
        assert np.array_equal(b.dist(q), ref)


def test_back_to_back_launches_without_wait():
    """A launch while the previous one is outstanding waits for it first:
    the later query set's results are exact, also through graph replay, and
    a solver launched twice reports the second source's distances."""
    from mlmq_tpds_withl3_b200 import Solver
    import torch
    g = HostGraph.grid(200, 150, seed=61)
    dg = DeviceGraph.upload(g)
    a, b_ = [0, 5, 77], [9000, 12, 29999]
    ref, _ = oracle_lib.sssp_many(g, a + b_)
    bs = BatchSolver(4, g.n, {"topup": 32})
    st = torch.cuda.Stream()
    for use_graph in (True, False):
        bs.launch([(dg, s) for s in a], use_graph=use_graph, stream=st.cuda_stream)
        bs.launch([(dg, s) for s in b_], use_graph=use_graph)
        bs.wait()
        for q in range(len(b_)):
            assert np.array_equal(bs.dist(q), ref[len(a) + q]), (use_graph, q)
    s = Solver(dg)
    s.launch(a[1], st.cuda_stream)
    s.launch(b_[1], None)
    s.wait()
    assert np.array_equal(s.dist(), ref[len(a) + 1])
