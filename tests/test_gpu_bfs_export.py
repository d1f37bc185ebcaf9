"""g5_bfs_export: the last search's result as one record (vertex, depth,
parent) per reached vertex, written by the kernel into pinned host memory or
a device buffer -- from the touched list after a one-block search, from a
scan of the parents otherwise -- equal to the search's own parent and depth
arrays; a too-small buffer is reported with the full count; exporting twice
gives the same records."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _records_from_arrays(bfs, with_depth):
    pred = bfs.pred.cpu().numpy()
    v = np.nonzero(pred != -1)[0]
    depth = bfs.depth.cpu().numpy()[v] if with_depth else np.full(len(v), -1)
    return v.astype(np.uint32), depth.astype(np.int32), pred[v]


def _sorted(rec):
    o = np.argsort(rec["vertex"], kind="stable")
    return rec["vertex"][o], rec["depth"][o], rec["parent"][o]


@pytest.fixture(scope="module")
def graph(cgt):
    g = cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), 16, 16 << 16)
    deg = np.diff(g.rowstarts.cpu().numpy())
    main = [r for r in cgt.generate_bfs_roots(g, 2, 3, 64) if g.in_main_component(r)][0]
    small = next(v for v in np.nonzero(deg > 0)[0] if not g.in_main_component(int(v)))
    return g, int(main), int(small)


@pytest.mark.parametrize("which", ["main", "small"])
@pytest.mark.parametrize("with_depth", [True, False])
def test_export_matches_search_arrays(cgt, graph, which, with_depth):
    g, main, small = graph
    root = main if which == "main" else small
    bfs = cgt.BfsState(g)
    for _ in range(2):  # the second query runs on a state reset to what the first touched
        cgt.oned_graph_bfs_reset(bfs, with_depth=True, g=g)
        st = cgt.oned_graph_bfs_query(g, bfs, root, with_depth=True)
        rec = cgt.oned_graph_bfs_export(g, bfs, with_depth=with_depth)
        assert len(rec) == st.reached
        want = _records_from_arrays(bfs, with_depth)
        for x, y in zip(_sorted(rec), want):
            assert np.array_equal(x, y)
        r0 = rec[rec["vertex"] == root]
        assert len(r0) == 1 and r0["parent"][0] == root and (r0["depth"][0] == 0 or not with_depth)
        if which == "small":  # the touched list: the root first, in the order reached
            assert rec["vertex"][0] == root
            assert np.all(np.diff(rec["depth"]) >= 0) or not with_depth
        # exported twice: the same records; into a device buffer: the same bytes' content
        again = cgt.oned_graph_bfs_export(g, bfs, with_depth=with_depth)
        assert np.array_equal(np.sort(again, order="vertex"), np.sort(rec, order="vertex"))
        dev = torch.empty(16 * g.nglobalverts, dtype=torch.uint8, device="cuda")
        d = cgt.oned_graph_bfs_export(g, bfs, with_depth=with_depth, out=dev).cpu().numpy().view(cgt.REACHED_DTYPE)
        assert np.array_equal(np.sort(d, order="vertex"), np.sort(rec, order="vertex"))


@pytest.mark.parametrize("which", ["main", "small"])
def test_query_export_in_one_call(cgt, graph, which):
    """g5_bfs_query_plan_export: the search and its export with one wait,
    the same records as a query followed by an export."""
    g, main, small = graph
    root = main if which == "main" else small
    a, b = cgt.BfsState(g), cgt.BfsState(g)
    for _ in range(2):
        cgt.oned_graph_bfs_reset(a, with_depth=True, g=g)
        cgt.oned_graph_bfs_reset(b, with_depth=True, g=g)
        st, rec = cgt.oned_graph_bfs_query_export(g, a, root, with_depth=True)
        assert len(rec) == st.reached
        for x, y in zip(_sorted(rec), _records_from_arrays(a, True)):
            assert np.array_equal(x, y)
        cgt.oned_graph_bfs_query(g, b, root, with_depth=True)
        ref = cgt.oned_graph_bfs_export(g, b, with_depth=True)
        # the same vertices at the same depths (parents may differ between two searches)
        assert np.array_equal(_sorted(rec)[0], _sorted(ref)[0]) and np.array_equal(_sorted(rec)[1], _sorted(ref)[1])


def test_export_reports_small_buffer(cgt, graph):
    g, main, _ = graph
    bfs = cgt.BfsState(g)
    cgt.oned_graph_bfs_reset(bfs, with_depth=True, g=g)
    st = cgt.oned_graph_bfs_query(g, bfs, main, with_depth=True)
    out = torch.empty(16 * 100, dtype=torch.uint8).pin_memory()
    cnt = torch.zeros(8, dtype=torch.uint8).pin_memory()
    rc = cgt.lib.g5_bfs_export(bfs.pred.data_ptr(), bfs.depth.data_ptr(), g.nglobalverts, bfs.work.data_ptr(),
                               bfs.work.numel(), out.data_ptr(), 100, cnt.data_ptr(), None)
    assert rc == -1 and b"capacity" in cgt.lib.g5_last_error()
    assert C.c_uint64.from_address(cnt.data_ptr()).value == st.reached
    # the records written are reached vertices with their parents
    rec = out.numpy().view(cgt.REACHED_DTYPE)
    pred = bfs.pred.cpu().numpy()
    assert np.array_equal(pred[rec["vertex"]], rec["parent"])
    # and a full export afterwards is complete
    full = cgt.oned_graph_bfs_export(g, bfs, with_depth=True)
    assert len(full) == st.reached
