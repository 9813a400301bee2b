"""Small graph fixtures for parity tests.

``supplement_fixture`` restates the reference's checked 2052-vertex graph
(scripts/multigpu/run_supplement_checks.py:25-40): a path chain 0..2049 with
asymmetric weights, a 512-way fan-out from vertex 0 and fan-in/fan-out through
vertex 1025, zero-weight 2-cycles 5<->6 and 1030<->1031, parallel arcs, and
isolated vertices 2050 and 2051.  The reference checks it from sources 0, 1030
and 2050 (run_supplement_checks.py:41).
"""
import numpy as np

from mlmq_tpds_withl3_b200 import HostGraph

SUPPLEMENT_SOURCES = (0, 1030, 2050)


def csr_from_adjacency(adj):
    row = [0]
    col, w = [], []
    for edges in adj:
        for v, wt in edges:
            col.append(v)
            w.append(wt)
        row.append(len(col))
    return (np.array(row, np.int32), np.array(col, np.int32), np.array(w, np.int32))


def supplement_fixture():
    n = 2052
    adj = [[] for _ in range(n)]
    for u in range(2049):
        adj[u].append((u + 1, 1 + u % 3))
        adj[u + 1].append((u, 1 + u % 5))
    for u in range(1, 513):
        adj[0].append((u, 1000 + u))
        adj[u].append((1025, u % 7))
        adj[1025].append((u, 2 + u % 5))
    for u in (5, 1030):
        adj[u].append((u + 1, 0))
        adj[u + 1].append((u, 0))
    row, col, w = csr_from_adjacency(adj)
    return HostGraph.from_csr(row, col, w, name="supplement2052")


def star_fixture(leaves=5000, hub_weight=7):
    """A hub with `leaves` out-arcs (warp-cooperative path) and a return arc
    from every leaf, plus a tail chain hanging off the last leaf."""
    n = leaves + 1 + 64
    adj = [[] for _ in range(n)]
    for i in range(1, leaves + 1):
        adj[0].append((i, hub_weight + (i * 37) % 1000))
        adj[i].append((0, 1 + i % 13))
    for i in range(leaves + 1, n):
        adj[i - 1].append((i, 3))
    row, col, w = csr_from_adjacency(adj)
    return HostGraph.from_csr(row, col, w, name=f"star{leaves}")


def components_fixture():
    """Two disconnected grids and a directed-only bridge: vertices of the
    second component are unreachable from the first."""
    a = HostGraph.grid(40, 40, seed=11)
    b = HostGraph.grid(30, 30, seed=12)
    na = a.n
    row = np.concatenate([a.row[:-1], b.row + a.m]).astype(np.int32)
    col = np.concatenate([a.col, b.col + na]).astype(np.int32)
    w = np.concatenate([a.w, b.w]).astype(np.int32)
    # one arc from the second component into the first (not back)
    row = row.copy()
    last = na + b.n - 1
    col = np.insert(col, row[last + 1], 0)
    w = np.insert(w, row[last + 1], 5)
    row[last + 1:] += 1
    return HostGraph.from_csr(row, col, w, name="components")


def golden_graphs():
    """name -> (HostGraph, sources) for the committed golden set."""
    return {
        "supplement2052": (supplement_fixture(), list(SUPPLEMENT_SOURCES)),
        "grid64": (HostGraph.grid(64, 64, seed=1), [0, 2080, 4095]),
        "knn3000": (HostGraph.knn(3000, seed=2), [0, 1500]),
        "rmat11": (HostGraph.rmat(11, seed=3), [0, 5]),
        "star2000": (star_fixture(2000), [0, 1999]),
        "components": (components_fixture(), [0, 1600 + 17]),
    }
