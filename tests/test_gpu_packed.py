"""Many graphs packed into one CSR and searched in one launch
(g5_csr_pack_append + g5_bfs_traverse_multi / g5_sssp_traverse_multi,
captured in a CUDA graph): every graph's slice equals that graph searched on
its own -- BFS depths and SSSP distances bit for bit, parent trees valid."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _np(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def packed(cgt):
    rng = np.random.default_rng(11)
    scales = rng.integers(4, 13, size=40).tolist()
    pk = cgt.pack_kronecker(scales, edgefactor=16, seed1_base=5, seed2=9)
    return scales, pk


def _single(cgt, scale, i):
    return cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(5 + i, 9), scale, 16 << scale)


def _canonical(rs, col, w):
    """Rows as sorted (column, weight bits) multisets: the CSR fill places a
    row's entries in atomic order, so two builds agree only up to order."""
    rows = np.repeat(np.arange(len(rs) - 1), np.diff(rs.astype(np.int64)))
    wb = w.view(np.uint32)
    o = np.lexsort((wb, col, rows))
    return col[o], wb[o]


def test_pack_layout(cgt, packed):
    scales, pk = packed
    assert pk.ngraphs == len(scales)
    assert list(pk.nverts) == [1 << s for s in scales]
    rs = _np(pk.g.rowstarts)
    for i in (0, 7, len(scales) - 1):
        g = _single(cgt, scales[i], i)
        sl = pk.graph_slice(i)
        base = rs[sl.start]
        assert np.array_equal(rs[sl.start:sl.stop + 1] - base, _np(g.rowstarts))
        e = g.nlocaledges
        pc, pw = _canonical(rs[sl.start:sl.stop + 1] - base, _np(pk.g.col[base:base + e]) - sl.start,
                            _np(pk.g.w[base:base + e]))
        gc, gw = _canonical(_np(g.rowstarts), _np(g.col), _np(g.w))
        assert np.array_equal(pc, gc) and np.array_equal(pw, gw)
        assert np.array_equal(_np(pk.g.light_deg[sl]), _np(g.light_deg))


@pytest.mark.parametrize("capture", [False, True])
def test_packed_batch_equals_single_searches(cgt, packed, capture):
    scales, pk = packed
    batch = cgt.PackedBatch(pk, delta=0.1, capture=capture)
    for _ in range(2):  # a replay gives the same answer again
        batch.run()
        batch.stream.synchronize()
        batch.check()
    depth, pred = _np(batch.bfs.depth), _np(batch.bfs.pred)
    dist, spred = _np(batch.sssp.dist), _np(batch.sssp.pred)
    for i in range(pk.ngraphs):
        g = _single(cgt, scales[i], i)
        sl = pk.graph_slice(i)
        r = int(pk.local_roots[i])
        bfs = cgt.BfsState(g)
        cgt.oned_graph_bfs_run(g, bfs, r)
        assert np.array_equal(depth[sl], _np(bfs.depth)), i
        # The packed parent tree, in the graph's own numbering, validates.
        lp = pred[sl].copy()
        lp[lp >= 0] -= sl.start
        bfs.pred.copy_(torch.as_tensor(lp, device=g.device))
        vw = cgt._val_work(g)
        d = cgt.bfs_compute_dist_from_pred(g, bfs, r)
        assert cgt.bfs_validate(g, r, bfs.pred, d, vw) == 0, i
        ss = cgt.SsspState(g)
        cgt.oned_graph_sssp_run(g, ss, r)
        assert np.array_equal(dist[sl].view(np.uint32), _np(ss.dist).view(np.uint32)), i
        sp = spred[sl].copy()
        sp[sp >= 0] -= sl.start
        assert cgt.sssp_validate(g, r, ss.dist, torch.as_tensor(sp, device=g.device), vw) == 0, i


def test_multi_root_edge_cases(cgt, oracle):
    """Repeated roots, an isolated root and two roots in one component:
    depths are the distance to the nearest root."""
    n = 64
    e = [(i, i + 1) for i in range(20)] + [(30, 31), (31, 32)]
    edges = torch.tensor(e, dtype=torch.int64, device="cuda")
    tg = cgt.TupleGraph(edges, torch.full((len(e),), 0.25, device="cuda"), len(e))
    g = cgt.oned_graph_from_tuple_graph(tg, n)
    roots = torch.tensor([0, 20, 20, 50, 31], dtype=torch.int64, device="cuda")
    bfs = cgt.BfsState(g)
    cgt.oned_graph_bfs_reset(bfs, True, g)
    cgt.oned_graph_bfs_traverse_multi(g, bfs, roots)
    d = _np(bfs.depth)
    want = np.full(n, -1)
    for v in range(21):
        want[v] = min(v, 20 - v)
    want[30], want[31], want[32], want[50] = 1, 0, 1, 0
    assert np.array_equal(d, want)
    assert cgt.bfs_stats(bfs).error_flags == 0
    ss = cgt.SsspState(g)
    cgt.oned_graph_sssp_reset(ss)
    cgt.oned_graph_sssp_traverse_multi(g, ss, roots)
    sd = _np(ss.dist)
    assert np.allclose(sd[want >= 0], 0.25 * want[want >= 0]) and np.all(sd[want < 0] == -1.0)
    with pytest.raises(ValueError):
        cgt.oned_graph_bfs_reset(bfs, True, g)
        cgt.oned_graph_bfs_traverse_multi(g, bfs, torch.tensor([n], dtype=torch.int64, device="cuda"))
        cgt.bfs_stats(bfs)
