"""The five synthetic workloads, seeded, with their source selection.

The reference measures on DIMACS road graphs that are not distributed with
it; these seeded generators stand in with the shapes, sizes and weight
distributions the measurement plan names:

  c1  512x512 4-neighbour grid, 10% of undirected edges dropped, w U{1000..100000},
      source 0, delta 200000
  c2  6.3M points uniform in the unit square, 3-NN symmetrised,
      w = round(1e6 * euclid) + 1, 5 seeded sources, delta autotuned
  c3  R-MAT scale 22, edge factor 16, (.57,.19,.19,.05), w U{1..2^20}
  c4  4896x4896 grid as c1, 64 seeded sources (batched)
  c5  grids 2^16..2^24 vertices + R-MAT 18/20/22 (served)
"""
import numpy as np

from .graph import HostGraph

SEED = 1


def largest_component_vertices(g):
    """Vertex ids of the largest weakly connected component."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components
    a = csr_matrix((np.ones(g.m, np.int8), g.col, g.row), shape=(g.n, g.n))
    _, labels = connected_components(a, directed=True, connection="weak")
    big = np.bincount(labels).argmax()
    return np.flatnonzero(labels == big)


def seeded_sources(g, count, seed=SEED, pool=None):
    """`count` distinct seeded random sources drawn from `pool` (default: the
    largest weakly connected component, so that each query reaches most of
    the graph as on the reference's connected road graphs)."""
    pool = largest_component_vertices(g) if pool is None else np.asarray(pool)
    rng = np.random.default_rng(seed)
    if count >= len(pool):
        return [int(v) for v in pool[:count]]
    return [int(v) for v in rng.choice(pool, size=count, replace=False)]


def probe_sources(g, timed, count=4, seed=SEED + 1000, pool=None):
    """`count` seeded sources for tuning, disjoint from the `timed` ones (a
    configuration is picked on sources the measurement does not use), drawn
    like seeded_sources from `pool` (default: the largest component)."""
    pool = largest_component_vertices(g) if pool is None else np.asarray(pool)
    pool = np.setdiff1d(pool, np.asarray(timed, dtype=pool.dtype))
    return seeded_sources(g, count, seed=seed, pool=pool)


def c1():
    return HostGraph.grid(512, 512, drop_p=0.10, wmin=1000, wmax=100000, seed=SEED), [0]


def c2(points=6_300_000, nsrc=5):
    g = HostGraph.knn(points, k=3, scale=1e6, seed=SEED)
    return g, seeded_sources(g, nsrc)


def c3(scale=22, nsrc=5):
    """Sources are drawn among the largest component's vertices with
    out-degree > 0 (a directed R-MAT vertex without out-arcs reaches only
    itself)."""
    g = HostGraph.rmat(scale, 16, 0.57, 0.19, 0.19, wmin=1, wmax=1 << 20, seed=SEED)
    return g, seeded_sources(g, nsrc, pool=c3_source_pool(g))


def c3_source_pool(g):
    comp = largest_component_vertices(g)
    return comp[np.diff(g.row)[comp] > 0]


def c4(side=4896, nsrc=64):
    g = HostGraph.grid(side, side, drop_p=0.10, wmin=1000, wmax=100000, seed=SEED)
    rng = np.random.default_rng(SEED)
    return g, [int(v) for v in rng.choice(g.n, size=nsrc, replace=False)]


def c5_graphs(max_log2=24, rmat_scales=(18, 20, 22)):
    """name -> HostGraph for the served mix."""
    out = {}
    for lg in range(16, max_log2 + 1, 2):
        side = 1 << (lg // 2)
        out[f"grid2^{lg}"] = HostGraph.grid(side, side, drop_p=0.10, wmin=1000, wmax=100000,
                                            seed=SEED + lg)
    for s in rmat_scales:
        out[f"rmat{s}"] = HostGraph.rmat(s, 16, 0.57, 0.19, 0.19, wmin=1, wmax=1 << 20,
                                         seed=SEED + 100 + s)
    return out


WORKLOADS = {"c1": c1, "c2": c2, "c3": c3, "c4": c4}
