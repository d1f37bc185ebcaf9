"""Canonical CSR build (g5_csr_fill_sorted, g5_csr_sort_rows, g5_csr_split_light,
g5_csr_dedupe_*): every row comes out sorted by (neighbour, weight bits) --
the reference fixtures' canonical hashes hold with no sorting on the host --
the build is the same on every run, the SSSP copy is each row stably split
into tiny | light | heavy parts, and the opt-in dedupe keeps the lightest
entry of each (row, neighbour) exactly as the oracle's restatement does.
Row lengths around every size class of the row sort (32/33, 256/257,
4096/4097 entries, and a hub of 150k) are covered by a synthetic graph."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from tests.golden.make_golden import canonical_csr, sha

pytestmark = pytest.mark.gpu


def _np(t):
    return t.cpu().numpy()


def _csr_host(g):
    return _np(g.rowstarts).view(np.uint64), _np(g.col).view(np.uint32), _np(g.w).view(np.uint32)


def test_canonical_rows_match_fixture_hashes(cgt, golden_dump):
    scale = golden_dump["scale"]
    seed = cgt.make_mrg_seed(2, 3)
    tg = cgt.generate_kronecker_range(seed, scale, 0, 16 << scale)
    for g in (cgt.oned_graph_from_tuple_graph(tg, 1 << scale, with_column64=True),
              cgt.oned_graph_from_kronecker(seed, scale, 16 << scale, with_column64=True)):
        rs, col, wb = _csr_host(g)
        assert sha(rs) == golden_dump["rowstarts_sha256"]
        assert sha(col, wb) == golden_dump["csr_canonical_sha256"]  # no canonicalisation step
        assert np.array_equal(_np(g.column), col.astype(np.int64))


def test_build_is_deterministic_and_split_is_stable(cgt):
    scale = 16
    seed = cgt.make_mrg_seed(7, 11)
    tg = cgt.generate_kronecker_range(seed, scale, 0, 16 << scale)
    a = cgt.oned_graph_from_tuple_graph(tg, 1 << scale)
    b = cgt.oned_graph_from_tuple_graph(tg, 1 << scale)
    for x, y in ((a.col, b.col), (a.w, b.w), (a.scol, b.scol), (a.sw, b.sw), (a.light_deg, b.light_deg)):
        assert torch.equal(x, y)
    rs, col, wb = _csr_host(a)
    scol, sw = _np(a.scol).view(np.uint32), _np(a.sw)
    ld, td = _np(a.light_deg).astype(np.int64), _np(a.tiny_deg).astype(np.int64)
    n = a.nglobalverts
    src = np.repeat(np.arange(n), np.diff(rs.astype(np.int64)))
    pos = np.arange(int(rs[-1])) - rs[src].astype(np.int64)
    light, tiny = np.float32(a.light_delta), np.float32(a.light_delta) / np.float32(30)
    cls = np.where(sw < tiny, 0, np.where(sw < light, 1, 2))
    want = np.where(pos < td[src], 0, np.where(pos < ld[src], 1, 2))
    assert np.array_equal(cls, want)
    # each part keeps the canonical order: sorting (row, part, key) changes nothing
    key = (scol.astype(np.uint64) << np.uint64(32)) | sw.view(np.uint32).astype(np.uint64)
    order = np.lexsort((key, cls, src))
    assert np.array_equal(order, np.arange(order.size))
    # and holds each row's entries
    c2, w2 = canonical_csr(rs, scol, sw)
    assert np.array_equal(c2, col) and np.array_equal(w2, wb)


def _dedupe_restated(rs, col, wb):
    """Keeps the first entry of each (row, neighbour) run of a canonical CSR."""
    n = rs.size - 1
    src = np.repeat(np.arange(n), np.diff(rs.astype(np.int64)))
    first = np.ones(col.size, bool)
    first[1:] = (src[1:] != src[:-1]) | (col[1:] != col[:-1])
    deg = np.bincount(src[first], minlength=n)
    rs2 = np.zeros(n + 1, np.uint64)
    rs2[1:] = np.cumsum(deg)
    return rs2, col[first], wb[first]


def test_dedupe_matches_restatement(cgt, oracle):
    scale = 14
    seed = cgt.make_mrg_seed(2, 3)
    n, m = 1 << scale, 16 << scale
    g = cgt.oned_graph_from_kronecker(seed, scale, m, dedupe=True, with_column64=True)
    oe, ow = oracle.generate_kronecker_range(np.array(seed, np.uint32), scale, 0, m)
    ors, ocol, ocw = oracle.csr_build(oe, ow, n)  # canonical rows, duplicates kept
    rs2, c2, w2 = _dedupe_restated(ors, ocol, ocw.view(np.uint32))
    rs, col, wb = _csr_host(g)
    assert np.array_equal(rs, rs2) and np.array_equal(col, c2) and np.array_equal(wb, w2)
    assert np.array_equal(_np(g.column), col.astype(np.int64))
    assert g.nlocaledges < ors[-1]  # Kronecker graphs have duplicate edges
    # a deduped graph still searches: BFS depths are those of the full graph
    full = cgt.oned_graph_from_kronecker(seed, scale, m)
    b1, b2 = cgt.BfsState(g), cgt.BfsState(full)
    r = cgt.generate_bfs_roots(full, 2, 3, 1)[0]
    cgt.oned_graph_bfs_run(g, b1, r)
    cgt.oned_graph_bfs_run(full, b2, r)
    assert torch.equal(b1.depth, b2.depth)


def test_row_size_classes(cgt):
    """Rows of every size class of the sort, duplicates with different
    weights included, against numpy's canonical order."""
    rng = np.random.default_rng(3)
    n = 1 << 18
    lens = [1, 2, 31, 32, 33, 100, 255, 256, 257, 1000, 4095, 4096, 4097, 9000, 150_000]
    edges, weights = [], []
    for i, L in enumerate(lens):
        hub = 1000 + i
        nb = rng.integers(200_000, n, size=L)
        nb[: L // 3] = nb[0]  # a run of duplicates
        edges.append(np.stack([np.full(L, hub), nb], 1))
        weights.append(rng.random(L, dtype=np.float32))
    e = np.concatenate(edges).astype(np.int64)
    wt = np.concatenate(weights)
    tg = cgt.TupleGraph(torch.from_numpy(e).cuda(), torch.from_numpy(wt).cuda(), e.shape[0])
    g = cgt.oned_graph_from_tuple_graph(tg, n, with_column64=True)
    rs, col, wb = _csr_host(g)
    # numpy: both directions of every edge, canonical rows
    src = np.concatenate([e[:, 0], e[:, 1]])
    dst = np.concatenate([e[:, 1], e[:, 0]])
    ww = np.concatenate([wt, wt]).view(np.uint32)
    order = np.lexsort((ww, dst, src))
    assert np.array_equal(col, dst[order].astype(np.uint32))
    assert np.array_equal(wb, ww[order])
    assert np.array_equal(np.diff(rs.astype(np.int64)), np.bincount(src, minlength=n))
    assert np.array_equal(_np(g.column), col.astype(np.int64))
    # sorting again changes nothing (g5_csr_sort_rows on canonical rows)
    work = cgt._sorted_work(n, g.nlocaledges, "cuda")
    c0, w0 = g.col.clone(), g.w.clone()
    assert cgt.lib.g5_csr_sort_rows(g.rowstarts.data_ptr(), n, g.nlocaledges, g.col.data_ptr(), g.w.data_ptr(),
                                    None, work.data_ptr(), work.numel(), None) == 0
    torch.cuda.synchronize()
    assert torch.equal(g.col, c0) and torch.equal(g.w, w0)


def test_fill_sorted_rejects_changed_edges(cgt):
    """Edges that do not match the row counts are reported, not written out
    of their rows."""
    dev = "cuda"
    e = torch.tensor([[0, 1], [1, 2], [2, 3]], dtype=torch.int64, device=dev)
    tg = cgt.TupleGraph(e, torch.ones(3, device=dev), 3)
    g = cgt.oned_graph_from_tuple_graph(tg, 4)
    e2 = torch.tensor([[0, 1], [1, 2], [0, 3]], dtype=torch.int64, device=dev)  # same count, other rows
    work = cgt._sorted_work(4, g.nlocaledges, dev)
    col = torch.empty(g.nlocaledges, dtype=torch.int32, device=dev)
    w = torch.empty(g.nlocaledges, dtype=torch.float32, device=dev)
    rc = cgt.lib.g5_csr_fill_sorted(e2.data_ptr(), tg.weights.data_ptr(), 3, 4, g.rowstarts.data_ptr(),
                                    g.nlocaledges, work.data_ptr(), work.numel(), col.data_ptr(), w.data_ptr(), None,
                                    None)
    assert rc == -1 and b"differ" in cgt.lib.g5_last_error()


def test_degree_order_copy(cgt):
    """g5_csr_degree_order: every row of the BFS copy holds the row's
    entries by decreasing neighbour degree, ties by index (rows of every
    size class, a hub of 150k included); BFS depths on it equal those on
    the canonical column and its parent trees validate."""
    rng = np.random.default_rng(4)
    n = 1 << 18
    lens = [3, 40, 300, 5000, 150_000]
    e = [np.stack([np.full(L, 7 + i), rng.integers(0, n, L)], 1) for i, L in enumerate(lens)]
    e.append(rng.integers(0, n, size=(400_000, 2)))
    e = np.concatenate(e).astype(np.int64)
    e = e[e[:, 0] != e[:, 1]]
    tg = cgt.TupleGraph(torch.from_numpy(e).cuda(), torch.ones(e.shape[0], device="cuda"), e.shape[0])
    g = cgt.oned_graph_from_tuple_graph(tg, n)
    cgt.oned_graph_bfs_order(g)
    rs = _np(g.rowstarts).astype(np.int64)
    col, bcol = _np(g.col).astype(np.int64), _np(g.bcol).astype(np.int64)
    deg = np.diff(rs)
    src = np.repeat(np.arange(n), deg)
    order = np.lexsort((col, -deg[col], src))  # numpy: rows by (-degree, index)
    assert np.array_equal(bcol, col[order])
    vw = cgt._val_work(g)
    bfs = cgt.BfsState(g)
    for r in (7, 11, int(e[-1, 0])):
        bcol_t, g.bcol = g.bcol, None
        cgt.oned_graph_bfs_run(g, bfs, r)
        want = bfs.depth.clone()
        g.bcol = bcol_t
        cgt.oned_graph_bfs_run(g, bfs, r)
        assert torch.equal(bfs.depth, want)
        d = cgt.bfs_compute_dist_from_pred(g, bfs, r)
        assert cgt.bfs_validate(g, r, bfs.pred, d, vw) == 0
