"""Graph transforms beside the solve path: BFS locality reordering
(reference graph_transform/reorder_gr.cu) and chain-shortcut augmentation G+
(reference SSSP/l3/l3_chain_shortcuts.h).

Both are pinned to the reference's own code: tests/golden/transforms.json holds
digests of what the reference's reorder_gr tool and chain builder produced on
every golden fixture (tests/golden/make_transforms.py), and when the
reference-built checkers are present in oracle/_ref/ the outputs are compared
with them directly as well.  The oracle then checks the property that makes
the transforms safe on the solve path: distances are unchanged (G+) or
permuted (reordering).
"""
import json
import os
import tempfile

import numpy as np
import pytest

import oracle_lib
from fixtures import csr_from_adjacency, golden_graphs
from mlmq_tpds_withl3_b200 import HostGraph
from golden.make_transforms import digest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "transforms.json")))
GRAPHS = golden_graphs()


@pytest.mark.parametrize("name", sorted(GOLD))
def test_reorder_matches_reference_digest(name):
    g, _ = GRAPHS[name]
    for root, want in GOLD[name]["reorder"].items():
        r, perm, inv = g.reorder_bfs(int(root))
        assert r.m == want["m"]
        assert digest(r.row, r.col, r.w, perm, inv) == want["sha256"], (name, root)


@pytest.mark.parametrize("name", sorted(GOLD))
def test_chain_shortcuts_match_reference_digest(name):
    g, _ = GRAPHS[name]
    for want in GOLD[name]["chain"].values():
        gp, st = g.chain_shortcuts(source=want["source"], cut=want["cut"])
        assert gp.m == want["m"]
        assert digest(gp.row, gp.col, gp.w) == want["sha256"], name
        assert [st[k] for k in ("chain_vertices", "shortcuts", "longest_walk",
                                "overflow_walks", "arcs_replaced")] == want["stats"]


def test_transforms_match_reference_checkers_directly():
    """Against oracle/_ref/ itself, on a graph that is not a golden fixture."""
    g = HostGraph.grid(96, 80, drop_p=0.25, seed=11)
    ref = oracle_lib.ref_chain_shortcuts(g, 17)
    if ref is None or not os.path.exists(oracle_lib.REORDER_BIN):
        pytest.skip("reference-built checkers not present")
    row, col, w, st = ref
    gp, mine = g.chain_shortcuts(source=17)
    assert np.array_equal(gp.row, row) and np.array_equal(gp.col, col)
    assert np.array_equal(gp.w, w)
    assert mine["shortcuts"] == st[1]
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "g.gr")
        g.write_gr(path)
        out, perm, inv = oracle_lib.ref_reorder_bfs(path, 5, td)
        rr = HostGraph.read_gr(out)
    r, p2, i2 = g.reorder_bfs(5)
    assert np.array_equal(perm, p2) and np.array_equal(inv, i2)
    assert np.array_equal(rr.row, r.row) and np.array_equal(rr.col, r.col)
    assert np.array_equal(rr.w, r.w)


@pytest.mark.parametrize("case", range(6))
def test_chain_shortcuts_equal_reference_on_seeded_graphs(case):
    """Seeded grids (many chains), kNN and R-MAT graphs with random sources
    and partition cuts: the pointer-jumping builder gives the reference
    builder's graph (oracle/_ref/libref_chain.so) byte for byte, statistics
    included."""
    rng = np.random.default_rng(100 + case)
    kind = case % 3
    if kind == 0:
        g = HostGraph.grid(int(rng.integers(40, 200)), int(rng.integers(40, 200)),
                           drop_p=float(rng.uniform(0.2, 0.6)), seed=int(rng.integers(1e6)))
    elif kind == 1:
        g = HostGraph.knn(int(rng.integers(2000, 20000)), k=int(rng.integers(1, 3)),
                          seed=int(rng.integers(1e6)))
    else:
        g = HostGraph.rmat(int(rng.integers(8, 12)), edge_factor=int(rng.integers(1, 4)),
                           seed=int(rng.integers(1e6)))
    src = int(rng.integers(g.n))
    cut = int(rng.integers(0, g.n + 1)) if case >= 3 else g.n
    ref = oracle_lib.ref_chain_shortcuts(g, src, cut)
    if ref is None:
        pytest.skip("reference-built checker not present")
    row, col, w, st = ref
    gp, mine = g.chain_shortcuts(source=src, cut=cut)
    assert np.array_equal(gp.row, row) and np.array_equal(gp.col, col)
    assert np.array_equal(gp.w, w)
    assert list(mine.values()) == [int(x) for x in st]


@pytest.mark.parametrize("name", ["grid64", "supplement2052", "components", "rmat11"])
def test_transforms_keep_distances(name):
    g, sources = GRAPHS[name]
    for src in sources:
        d0, _ = oracle_lib.sssp_i32(g, src)
        gp, _ = g.chain_shortcuts(source=src)
        d1, _ = oracle_lib.sssp_i32(gp, src)
        assert np.array_equal(d0, d1)
        r, perm, inv = g.reorder_bfs(src)
        assert perm[0] == src and inv[src] == 0
        d2, _ = oracle_lib.sssp_i32(r, int(inv[src]))
        assert np.array_equal(d2[inv], d0)


def test_chain_shortcuts_path_known_answer():
    """Bidirectional path 0-1-2-3-4: 1, 2 and 3 are chain vertices, so each end
    gets one shortcut to the other end with the summed weight."""
    adj = [[(1, 2)], [(0, 3), (2, 5)], [(1, 7), (3, 11)], [(2, 13), (4, 17)], [(3, 19)]]
    row, col, w = csr_from_adjacency(adj)
    g = HostGraph.from_csr(row, col, w)
    gp, st = g.chain_shortcuts(source=0)
    assert st["chain_vertices"] == 3 and st["shortcuts"] == 2 and st["longest_walk"] == 4
    assert list(gp.col[gp.row[0]:gp.row[1]]) == [4, 1]
    assert list(gp.w[gp.row[0]:gp.row[1]]) == [2 + 5 + 11 + 17, 2]
    assert list(gp.col[gp.row[4]:gp.row[5]]) == [0, 3]
    assert list(gp.w[gp.row[4]:gp.row[5]]) == [19 + 13 + 7 + 3, 19]


def test_reorder_bfs_order_and_unreached_tail():
    """Discovery order of a queue BFS scanning arcs in CSR order; vertices the
    BFS never reaches follow in ascending id."""
    adj = [[(2, 1), (1, 1)], [(3, 1)], [(3, 1)], [], [(0, 1)], []]
    row, col, w = csr_from_adjacency(adj)
    g = HostGraph.from_csr(row, col, w)
    _, perm, inv = g.reorder_bfs(0)
    assert list(perm) == [0, 2, 1, 3, 4, 5]
    assert list(inv[perm]) == list(range(6))


def test_transform_argument_errors():
    g = HostGraph.grid(8, 8)
    from mlmq_tpds_withl3_b200._lib import MlmqError
    with pytest.raises(MlmqError):
        g.reorder_bfs(64)
    with pytest.raises(MlmqError):
        g.chain_shortcuts(source=-1)
    with pytest.raises(MlmqError):
        g.chain_shortcuts(source=0, cut=65)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GOLD))
def test_gpu_reorder_matches_reference_digest(name):
    """BFS reordering as a device preprocessing step: the reference tool's
    output (golden digests made by graph_transform/reorder_gr.cu) byte for
    byte, for every golden fixture and root."""
    g, _ = GRAPHS[name]
    for root, want in GOLD[name]["reorder"].items():
        r, perm, inv = g.reorder_bfs_gpu(int(root))
        assert r.m == want["m"]
        assert digest(r.row, r.col, r.w, perm, inv) == want["sha256"], (name, root)


@pytest.mark.gpu
def test_gpu_reorder_equals_host_on_large_graphs():
    """Large road-like, kNN and R-MAT graphs (hubs, unreached vertices, many
    levels): the device reordering equals the host one, and the reordered
    graph solves to the permuted distances on the GPU."""
    from mlmq_tpds_withl3_b200 import DeviceGraph, Solver
    for g, root in ((HostGraph.grid(700, 500, drop_p=0.3, seed=61), 1234),
                    (HostGraph.knn(300000, seed=62), 77),
                    (HostGraph.rmat(17, seed=63), 5)):
        h, hp, hi = g.reorder_bfs(root)
        d, dp, di = g.reorder_bfs_gpu(root)
        assert np.array_equal(hp, dp) and np.array_equal(hi, di), g
        assert np.array_equal(h.row, d.row) and np.array_equal(h.col, d.col)
        assert np.array_equal(h.w, d.w)
        ref, _ = oracle_lib.sssp_i32(g, root)
        got = Solver(DeviceGraph.upload(d)).solve(int(di[root])).dist()
        assert np.array_equal(got[di], ref), g
