"""Resets that undo only what the last search wrote (g5_bfs_reset_touched,
g5_sssp_reset_touched): after every reset the outputs and the visited bitmap
are exactly as a full reset leaves them, whatever ran before -- one-block
searches, grid searches, searches with other output arrays -- and searches
after such resets give the results of searches on fresh states."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _np(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def g16(cgt):
    return cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), 16, 16 << 16)


def _roots(cgt, g):
    rs = _np(g.rowstarts)
    n = g.nglobalverts
    main = (np.asarray(g.main_bits, np.uint32)[np.arange(n) >> 5] >> (np.arange(n) & 31).astype(np.uint32)) & 1
    small = np.nonzero((main == 0) & (rs[1:] > rs[:-1]))[0][:4].tolist()
    big = cgt.generate_bfs_roots(g, 2, 3, 3)
    assert small and big
    return small, big


def _visited(cgt, g, bfs):
    bits = torch.empty((g.nglobalverts + 31) // 32, dtype=torch.int32, device="cuda")
    assert cgt.lib.g5_bfs_visited_bitmap(bfs.work.data_ptr(), bfs.work.numel(), g.nglobalverts, bits.data_ptr(),
                                         None) == 0
    return _np(bits)


def test_bfs_touched_reset_leaves_a_clean_state(cgt, oracle, g16):
    g = g16
    small, big = _roots(cgt, g)
    iso = _np(g.isolated)
    bfs = cgt.BfsState(g)
    other_depth = torch.empty_like(bfs.depth)
    rs, col = _np(g.rowstarts).view(np.uint64), _np(g.col).view(np.uint32)
    seq = [(small[0], True), (small[1], True), (big[0], False), (small[2], True), (small[0], False),
           (big[1], True), (small[3], True), (small[1], True)]
    for i, (r, with_depth) in enumerate(seq):
        cgt.oned_graph_bfs_reset(bfs, with_depth=with_depth, g=g)
        assert bfs.was_reset
        torch.cuda.synchronize()
        assert (_np(bfs.pred) == -1).all(), (i, r)
        if with_depth:
            assert (_np(bfs.depth) == -1).all(), (i, r)
        assert np.array_equal(_visited(cgt, g, bfs), iso), (i, r)
        cgt.oned_graph_bfs_traverse(g, bfs, r, with_depth=with_depth)
        st = cgt.bfs_stats(bfs)
        _, od = oracle.bfs(rs, col, g.nglobalverts, r)
        assert st.reached == int((od != -1).sum()), (i, r)
        if with_depth:
            assert np.array_equal(_np(bfs.depth).astype(np.int64), od), (i, r)
    # A reset given another depth array clears that array in full.
    other_depth.fill_(5)
    d0 = bfs.depth
    bfs.depth = other_depth
    cgt.oned_graph_bfs_reset(bfs, with_depth=True, g=g)
    torch.cuda.synchronize()
    assert (_np(other_depth) == -1).all()
    bfs.depth = d0
    assert cgt.lib.g5_bfs_reset(g.nglobalverts, bfs.pred.data_ptr(), bfs.depth.data_ptr(), g.isolated.data_ptr(),
                                bfs.work.data_ptr(), bfs.work.numel(), None) == 0
    # A reset after a search that started from another visited bitmap
    # restores the bitmap in full (and pred and depth from the list).
    cgt.oned_graph_bfs_traverse(g, bfs, small[0], with_depth=True)
    cgt.oned_graph_bfs_reset(bfs, with_depth=True, g=None)
    torch.cuda.synchronize()
    assert (_visited(cgt, g, bfs) == 0).all()
    assert (_np(bfs.pred) == -1).all() and (_np(bfs.depth) == -1).all()


def test_sssp_touched_reset_leaves_a_clean_state(cgt, oracle, g16):
    g = g16
    small, big = _roots(cgt, g)
    rs, col, w = _np(g.rowstarts).view(np.uint64), _np(g.col).view(np.uint32), _np(g.w)
    s = cgt.SsspState(g)
    fresh = cgt.SsspState(g)
    seq = [small[0], small[1], big[0], small[2], big[1], small[3], small[0]]
    for i, r in enumerate(seq):
        cgt.oned_graph_sssp_reset(s)
        torch.cuda.synchronize()
        assert (_np(s.dist) == -1.0).all() and (_np(s.pred) == -1).all(), (i, r)
        cgt.oned_graph_sssp_traverse(g, s, r)
        cgt.sssp_status(s)
        cgt.oned_graph_sssp_run(g, fresh, r)  # full reset first
        assert np.array_equal(_np(s.dist).view(np.uint32), _np(fresh.dist).view(np.uint32)), (i, r)
        assert np.array_equal(_np(s.pred), _np(fresh.pred)), (i, r)
        od, _ = oracle.sssp(rs, col, w, g.nglobalverts, r)
        assert np.array_equal(_np(s.dist).view(np.uint32), od.view(np.uint32)), (i, r)
    # Outputs the last search did not write sparsely are prefilled in full.
    d2, p2 = torch.full_like(s.dist, 3.0), torch.full_like(s.pred, 3)
    assert cgt.lib.g5_sssp_reset_touched(s.max_nlocalverts, d2.data_ptr(), p2.data_ptr(), s.work.data_ptr(),
                                         s.work.numel(), None) == 0
    torch.cuda.synchronize()
    assert (_np(d2) == -1.0).all() and (_np(p2) == -1).all()


def test_touched_reset_costs_reached_not_n(cgt, g16):
    """After a one-block search the touched reset is one small launch: at
    least twice as fast as the full reset on a graph of 2^24 vertices (whose
    pred array alone is 134 MB)."""
    g = cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), 24, 16 << 24)
    small, _ = _roots(cgt, g)
    bfs = cgt.BfsState(g)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    full, touched = [], []
    for _ in range(5):
        torch.cuda._sleep(200_000)  # both resets queued before the device reaches them
        ev[0].record()
        assert cgt.lib.g5_bfs_reset(g.nglobalverts, bfs.pred.data_ptr(), None, g.isolated.data_ptr(),
                                    bfs.work.data_ptr(), bfs.work.numel(), None) == 0
        ev[1].record()
        cgt.oned_graph_bfs_traverse(g, bfs, small[0], with_depth=False)
        ev[2].record()
        assert cgt.lib.g5_bfs_reset_touched(g.nglobalverts, bfs.pred.data_ptr(), None, g.isolated.data_ptr(),
                                            bfs.work.data_ptr(), bfs.work.numel(), None) == 0
        ev[3].record()
        torch.cuda.synchronize()
        full.append(ev[0].elapsed_time(ev[1]))
        touched.append(ev[2].elapsed_time(ev[3]))
    assert (_np(bfs.pred) == -1).all()
    assert min(touched) * 2 < min(full), (touched, full)
