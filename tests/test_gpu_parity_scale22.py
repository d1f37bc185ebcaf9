"""Parity at SCALE 22, edgefactor 16 (4.2M vertices, 67M edges): the GPU path
and the oracle each build the graph from the same seeds, and are compared
bit for bit -- edge list and weights, CSR (rows in canonical order), the
runner's roots, BFS depth arrays for the runner's first roots and every one
of its 64 roots outside the main component (the 2-vertex-component root that
sets the harmonic mean among them), SSSP distance bits from a main-component
and a small-component source, and the runner's TEPS edge counts."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SCALE = 22


def _np(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def s22(cgt, oracle):
    n, m = 1 << SCALE, 16 << SCALE
    seed = cgt.make_mrg_seed(2, 3)
    tg = cgt.generate_kronecker_range(seed, SCALE, 0, m)
    oe, ow = oracle.generate_kronecker_range(np.array(seed, np.uint32), SCALE, 0, m)
    edges_equal = np.array_equal(_np(tg.edges).view(np.uint64).reshape(-1), oe.reshape(-1))
    weights_equal = np.array_equal(_np(tg.weights).view(np.uint32), ow.view(np.uint32))
    g = cgt.oned_graph_from_tuple_graph(tg, n)
    del tg
    torch.cuda.empty_cache()
    ors, ocol, ocw = oracle.csr_build(oe, ow, n)
    del oe, ow
    return dict(g=g, n=n, ors=ors, ocol=ocol, ocw=ocw, edges_equal=edges_equal, weights_equal=weights_equal)


def _canonical_gpu(g):
    """The GPU CSR's rows sorted by (dst, weight bits), sorted on the GPU."""
    rs = g.rowstarts
    n = g.nglobalverts
    src = torch.repeat_interleave(torch.arange(n, device=rs.device), rs[1:] - rs[:-1])
    wb = g.w.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    o1 = torch.sort(wb, stable=True).indices
    key = (src[o1] << SCALE) | g.col[o1].to(torch.int64)
    o2 = torch.sort(key, stable=True).indices
    order = o1[o2]
    return _np(g.col[order]).view(np.uint32), _np(g.w[order]).view(np.uint32)


def test_generation_and_csr_bit_exact(s22):
    assert s22["edges_equal"] and s22["weights_equal"]
    g = s22["g"]
    assert np.array_equal(_np(g.rowstarts).view(np.uint64), s22["ors"])
    col, wb = _canonical_gpu(g)
    assert np.array_equal(col, s22["ocol"]) and np.array_equal(wb, s22["ocw"].view(np.uint32))


def test_roots_bfs_depths_and_edge_counts(cgt, oracle, s22):
    g, n = s22["g"], s22["n"]
    roots = cgt.generate_bfs_roots(g, 2, 3, 64)
    assert roots == oracle.generate_bfs_roots(s22["ors"], n, 2, 3, 64).tolist()
    small = [r for r in roots if not g.in_main_component(r)]
    assert small, "the runner's SCALE 22 roots include a small-component root"
    bfs, vw = cgt.BfsState(g), cgt._val_work(g)
    for r in roots[:6] + small:
        cgt.oned_graph_bfs_run(g, bfs, r)
        opred, odepth = oracle.bfs(s22["ors"], s22["ocol"], n, r)
        assert np.array_equal(_np(bfs.depth).astype(np.int64), odepth), r
        dist = cgt.bfs_compute_dist_from_pred(g, bfs, r)
        assert cgt.bfs_validate(g, r, bfs.pred, dist, vw) == 0, r
        assert cgt.edge_count(g, bfs.pred, vw) == oracle.edge_count(s22["ors"], s22["ocol"], n, opred), r


def test_sssp_distance_bits(cgt, oracle, s22):
    g, n = s22["g"], s22["n"]
    roots = cgt.generate_bfs_roots(g, 2, 3, 64)
    small = [r for r in roots if not g.in_main_component(r)]
    s, vw = cgt.SsspState(g), cgt._val_work(g)
    for r in (roots[0], small[0]):
        cgt.oned_graph_sssp_run(g, s, r)
        cgt.sssp_status(s)
        od, _ = oracle.sssp(s22["ors"], s22["ocol"], s22["ocw"], n, r)
        assert np.array_equal(_np(s.dist).view(np.uint32), od.view(np.uint32)), r
        assert cgt.sssp_validate(g, r, s.dist, s.pred, vw) == 0, r
