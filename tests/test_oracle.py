"""The oracle pinned against the golden vectors made by the reference's own
code (tests/golden/make_golden.py), and against the reference's compiled
sssp_sequential when it is present."""
import json
import os

import numpy as np
import pytest

import oracle_lib
from fixtures import golden_graphs
from mlmq_tpds_withl3_b200 import HostGraph

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def cases():
    for name, entry in sorted(manifest().items()):
        for src in sorted(entry["sources"], key=int):
            yield name, int(src)


@pytest.mark.parametrize("name,src", list(cases()))
def test_oracle_i32_matches_golden(name, src):
    entry = manifest()[name]
    g = HostGraph.read_gr(os.path.join(GOLDEN, entry["file"]))
    gold = np.fromfile(os.path.join(GOLDEN, entry["sources"][str(src)]["file"]), dtype=np.int32)
    d, work = oracle_lib.sssp_i32(g, src)
    assert np.array_equal(d, gold)
    assert work == entry["sources"][str(src)]["total_work"]


@pytest.mark.parametrize("name,src", list(cases()))
def test_oracle_i64_matches_golden(name, src):
    entry = manifest()[name]
    g = HostGraph.read_gr(os.path.join(GOLDEN, entry["file"]))
    gold = np.fromfile(os.path.join(GOLDEN, entry["sources"][str(src)]["file"]), dtype=np.int32)
    d, reached, mx = oracle_lib.sssp_i64(g, src)
    assert np.array_equal(d, gold)
    assert reached == entry["sources"][str(src)]["reached"]
    assert mx == entry["sources"][str(src)]["max_distance"]


def test_fixture_files_are_the_fixture_graphs():
    """The committed .gr files are exactly what fixtures.py builds."""
    for name, (g, _) in golden_graphs().items():
        back = HostGraph.read_gr(os.path.join(GOLDEN, f"{name}.gr"))
        assert back.n == g.n and back.m == g.m
        assert np.array_equal(back.row, g.row)
        assert np.array_equal(back.col, g.col)
        assert np.array_equal(back.w, g.w)


def test_supplement_known_answers():
    """Known answers of the reference's fixture: 2050 and 2051 unreachable
    from 0, zero-weight 2-cycles, the fan-in through 1025."""
    g = HostGraph.read_gr(os.path.join(GOLDEN, "supplement2052.gr"))
    d, _ = oracle_lib.sssp_i32(g, 0)
    assert d[2050] == oracle_lib.INT_MAX and d[2051] == oracle_lib.INT_MAX
    assert d[5] == d[6]
    d2, _ = oracle_lib.sssp_i32(g, 2050)
    assert d2[2050] == 0 and (d2 == oracle_lib.INT_MAX).sum() == g.n - 1
    d3, _ = oracle_lib.sssp_i32(g, 1030)
    assert d3[1031] == 0


@pytest.mark.skipif(oracle_lib.reference() is None, reason="reference checker not built")
def test_oracle_matches_reference_binary_on_synthetic():
    for g in (HostGraph.grid(96, 80, seed=5), HostGraph.knn(5000, seed=6),
              HostGraph.rmat(12, seed=7)):
        for src in (0, g.n // 3):
            d, work = oracle_lib.sssp_i32(g, src)
            r, rwork = oracle_lib.ref_sequential(g, src)
            assert np.array_equal(d, r)
            assert work == rwork


def test_oracle_many_matches_single():
    g = HostGraph.grid(50, 50, seed=9)
    srcs = [0, 7, 1234, 2499]
    d, work = oracle_lib.sssp_many(g, srcs, threads=3)
    for k, s in enumerate(srcs):
        one, w1 = oracle_lib.sssp_i32(g, s)
        assert np.array_equal(d[k], one) and work[k] == w1


def test_oracle_rejects_overflow():
    # a 3-vertex path whose second hop exceeds INT_MAX
    g = HostGraph.from_csr([0, 1, 2, 2], [1, 2], [2**31 - 10, 100])
    with pytest.raises(RuntimeError):
        oracle_lib.sssp_i32(g, 0)
    with pytest.raises(RuntimeError):
        oracle_lib.sssp_i64(g, 0)


def test_digest_statements_agree_and_separate_results():
    """The served-result fingerprint, stated three times (oracle C, numpy,
    the library's host function), gives one value per distance array, and
    differs when one distance differs."""
    from mlmq_tpds_withl3_b200._lib import dist_digest
    g, _ = golden_graphs()["supplement2052"]
    d, _ = oracle_lib.sssp_i32(g, 0)
    a = oracle_lib.digest(d)
    assert a == oracle_lib.digest_numpy(d) == dist_digest(d)
    e = d.copy()
    e[1025] += 1
    assert oracle_lib.digest(e) != a
    f = d.copy()
    f[[3, 4]] = f[[4, 3]]  # the same values at other vertices
    if f[3] != f[4]:
        assert oracle_lib.digest(f) != a
    # the digest of many sources equals the digests of the full results
    srcs = [0, 1030, 2050]
    dg, work, reached = oracle_lib.sssp_digest_many(g, srcs, threads=2)
    full, works = oracle_lib.sssp_many(g, srcs)
    assert [int(x) for x in dg] == [oracle_lib.digest(r) for r in full]
    assert list(work) == list(works)
    assert list(reached) == [int((r != oracle_lib.INT_MAX).sum()) for r in full]
