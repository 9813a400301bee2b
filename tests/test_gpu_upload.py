"""The device arc array after upload: each vertex's arcs are a permutation of
its input arcs, sorted by weight (the order the light/heavy split and the
inline tile arcs rely on).  Skewed graphs (a vertex above 1024 arcs) take
the radix-sort path of the upload, graphs of small degrees the segmented
sort; both are checked, as is the caller-owned device CSR path of the
reference entry points (SS/SSSP/sssp_run.cu:676, sssp_init)."""
import numpy as np
import pytest
import torch

from mlmq_tpds_withl3_b200 import DeviceGraph, HostGraph

pytestmark = pytest.mark.gpu


def _check_arcs(g, col, w):
    row = np.asarray(g.row, np.int64)
    hc, hw = np.asarray(g.col, np.int32), np.asarray(g.w, np.int32)
    vid = np.repeat(np.arange(g.n), np.diff(row))
    same = vid[1:] == vid[:-1]
    assert np.all(w[1:][same] >= w[:-1][same]), "a vertex's arcs are not sorted by weight"
    a = np.lexsort((col, w, vid))
    b = np.lexsort((hc, hw, vid))
    assert np.array_equal(col[a], hc[b]) and np.array_equal(w[a], hw[b]), \
        "a vertex's arcs are not a permutation of its input arcs"


@pytest.mark.parametrize("kind", ["rmat", "rmat_wide_weights", "grid", "rmat_ranges", "grid_ranges"])
def test_uploaded_arcs_are_each_vertex_arcs_sorted_by_weight(kind):
    # *_ranges: above 8M arcs the upload copies and sorts the graph in
    # ranges of vertices, each sorted while the next is copied
    if kind == "rmat":
        g = HostGraph.rmat(16, 16, seed=5)
    elif kind == "rmat_wide_weights":
        g = HostGraph.rmat(15, 16, wmin=0, wmax=(1 << 31) - 2, seed=6)
    elif kind == "rmat_ranges":
        g = HostGraph.rmat(20, 16, seed=9)
        assert g.m >= 8 << 20
    elif kind == "grid_ranges":
        g = HostGraph.grid(1600, 1500, seed=10)
        assert g.m >= 8 << 20
    else:
        g = HostGraph.grid(300, 200, seed=7)
    dg = DeviceGraph.upload(g)
    if kind.startswith("rmat"):
        assert dg.pieces > 0  # a vertex above 1024 arcs: the radix-sort path
    else:
        assert dg.pieces == 0
    col, w = dg.arcs()
    _check_arcs(g, col, w)
    dg.close()


def test_wrapped_device_csr_arcs_sorted_and_inputs_untouched():
    g = HostGraph.rmat(15, 16, seed=8)
    d_row = torch.from_numpy(np.asarray(g.row, np.int32)).cuda()
    d_col = torch.from_numpy(np.asarray(g.col, np.int32)).cuda()
    d_w = torch.from_numpy(np.asarray(g.w, np.int32)).cuda()
    dg = DeviceGraph.wrap_device(g.n, g.m, d_row.data_ptr(), d_col.data_ptr(), d_w.data_ptr())
    col, w = dg.arcs()
    _check_arcs(g, col, w)
    # the caller's arrays are read, never reordered
    assert np.array_equal(d_col.cpu().numpy(), np.asarray(g.col, np.int32))
    assert np.array_equal(d_w.cpu().numpy(), np.asarray(g.w, np.int32))
    dg.close()
