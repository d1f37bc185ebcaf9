"""The bottom-up levels' first-neighbour probe (g5_bfs_params.top from
g5_bfs_first_neighbours): the array holds each row's first entry of the
BFS's degree-ordered column, and searches with and without it choose the
same parent for every vertex (the probe is the row scan's first step)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_first_neighbour_probe_same_parents(cgt):
    g = cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), 18, 16 << 18)
    n = g.nglobalverts
    assert g.btop is not None and g.bcol is not None
    rs = g.rowstarts.cpu().numpy().astype(np.int64)
    bc = g.bcol.cpu().numpy()
    top = g.btop.cpu().numpy().view(np.uint32)
    full = rs[:-1] < rs[1:]
    assert np.array_equal(top[full], bc[rs[:-1][full]].view(np.uint32))
    assert np.all(top[~full] == n)
    roots = [r for r in cgt.generate_bfs_roots(g, 2, 3, 64) if g.in_main_component(r)][:4]
    a, b = cgt.BfsState(g), cgt.BfsState(g)
    for mode in (0, 2):  # direction-optimizing; bottom-up from level 1 on
        for r in roots:
            outs = []
            for st, use_top in ((a, True), (b, False)):
                cgt.oned_graph_bfs_reset(st, True, g)
                p = cgt.BfsParams(14.0, 24.0, mode, 0)
                if use_top:
                    p.top = g.btop.data_ptr()
                rc = cgt.lib.g5_bfs_traverse(g.rowstarts.data_ptr(), g.bcol.data_ptr(), n, int(r), st.pred.data_ptr(),
                                             st.depth.data_ptr(), st.work.data_ptr(), st.work.numel(), C.byref(p),
                                             None)
                assert rc == 0, cgt.lib.g5_last_error()
                torch.cuda.synchronize()
                outs.append((st.pred.clone(), st.depth.clone(), cgt.bfs_stats(st).bottom_up_levels))
            assert outs[0][2] > 0  # bottom-up levels ran
            assert torch.equal(outs[0][1], outs[1][1])
            if mode == 2:  # every level after the first bottom-up: the parents are determined
                assert torch.equal(outs[0][0], outs[1][0])
    vw = cgt._val_work(g)
    d = cgt.bfs_compute_dist_from_pred(g, a, int(roots[-1]))
    assert cgt.bfs_validate(g, int(roots[-1]), a.pred, d, vw) == 0
