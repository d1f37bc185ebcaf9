"""Batched BFS (g5_msbfs_*, up to 256 roots per search) against the
reference's depth arrays, the oracle and the single-root BFS.  Depths are
integers: every root's array must be identical."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from tests.conftest import load_golden, GOLDEN
from tests.golden.make_golden import sha

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kron(cgt):
    seed = cgt.make_mrg_seed(2, 3)
    return {s: cgt.oned_graph_from_kronecker(seed, s, 16 << s) for s in (12, 14, 16)}


def _depths(cgt, ms):
    d = cgt.msbfs_depths_u8(ms).cpu().numpy().astype(np.int64)
    d[d == 255] = -1
    return d


def _host_csr(g):
    return g.rowstarts.cpu().numpy().view(np.uint64), g.col.cpu().numpy().view(np.uint32)


def test_msbfs_matches_reference_depths_scale12(cgt, kron):
    """The 64 runner roots of the SCALE 12 fixture in one batch: each depth
    array equals the reference's own (bfs_compute_dist_from_pred)."""
    g = kron[12]
    ref = np.load(f"{GOLDEN}/ref_s12_depth.npz")["depth"].astype(np.int64)
    roots = load_golden("ref_s12.json")["roots"]
    ms = cgt.MsBfsState(g)
    st = cgt.msbfs_run(g, ms, roots)
    assert st.error_flags == 0 and st.nroots == len(roots)
    d = _depths(cgt, ms)
    assert d.shape == ref.shape
    for i in range(len(roots)):
        assert np.array_equal(d[i], ref[i]), i
    assert st.pairs_reached == int((ref != -1).sum())


def test_msbfs_matches_reference_hashes_scale14(cgt, kron):
    g = kron[14]
    fx = load_golden("ref_s14.json")
    roots = [pr["root"] for pr in fx["per_root"]]
    ms = cgt.MsBfsState(g)
    cgt.msbfs_run(g, ms, roots)
    d = _depths(cgt, ms)
    for i, pr in enumerate(fx["per_root"]):
        assert sha(d[i]) == pr["depth_sha256"], pr["root"]
        assert int((d[i] != -1).sum()) == pr["reached"]
        assert int(d[i].max()) == pr["max_depth"]


@pytest.mark.parametrize("params", [None, (4.0, 1, 0, 0), (4.0, 2, 0, 0), (4.0, 2, 1, 0), (4.0, 2, 2, 0),
                                    (1.0, 0, 0, 0), (64.0, 0, 0, 0), (4.0, 0, 0, 1), (4.0, 0, 0, 3)])
def test_msbfs_256_roots_equal_single_searches(cgt, oracle, kron, params):
    """256 roots (repeats and an isolated vertex among them) on SCALE 16:
    automatic, top-down-only and pull-only directions, with and without the
    frontier-bitmap test, on any grid: every depth array equals the oracle's
    single-root BFS and the library's own g5_bfs_run depth."""
    g = kron[16]
    n = g.nglobalverts
    rs, col = _host_csr(g)
    deg = np.diff(rs.astype(np.int64))
    rng = np.random.default_rng(7)
    roots = rng.choice(np.nonzero(deg > 0)[0], 250, replace=False).tolist()
    roots += [roots[0], roots[5], int(np.nonzero(deg == 0)[0][0]), int(np.argmax(deg)), roots[17], 0]
    assert len(roots) == 256
    ms = cgt.MsBfsState(g)
    p = cgt.MsBfsParams(*params) if params is not None else None
    st = cgt.msbfs_run(g, ms, roots, p)
    assert st.error_flags == 0
    d = _depths(cgt, ms)
    check = range(256) if params is None else list(range(0, 256, 9)) + [250, 251, 252, 253, 255]
    for i in check:
        _, od = oracle.bfs(rs, col, n, roots[i])
        assert np.array_equal(d[i], od), (i, roots[i])
    if params is None:
        bfs = cgt.BfsState(g)
        for i in (0, 3, 250, 252, 253):
            cgt.oned_graph_bfs_run(g, bfs, roots[i])
            assert np.array_equal(d[i], bfs.depth.cpu().numpy().astype(np.int64)), i
        assert st.pairs_reached == int((d != -1).sum())
        one = cgt.msbfs_depth(ms, 253).cpu().numpy()
        assert np.array_equal(one.astype(np.int64), d[253])


def test_msbfs_reuse_and_batch_sizes(cgt, oracle, kron):
    """One workspace, consecutive searches of 1, 256 and 33 roots: each
    result is the same as on a fresh workspace."""
    g = kron[14]
    n = g.nglobalverts
    rs, col = _host_csr(g)
    roots = cgt.generate_bfs_roots(g, 2, 3, 64)
    ms = cgt.MsBfsState(g)
    for batch in ([roots[3]], (roots * 4)[:256], roots[10:43]):
        st = cgt.msbfs_run(g, ms, batch)
        assert st.error_flags == 0
        d = _depths(cgt, ms)
        assert d.shape == (len(batch), n)
        for i in {0, len(batch) // 2, len(batch) - 1}:
            _, od = oracle.bfs(rs, col, n, batch[i])
            assert np.array_equal(d[i], od)
    fresh = cgt.MsBfsState(g)
    cgt.msbfs_run(g, fresh, roots[10:43])
    assert np.array_equal(_depths(cgt, fresh), d)


def _small_graph(cgt):
    # A 120-vertex path, a star, a triangle, a self-loop, isolated vertices.
    n = 1000
    e = [(i, i + 1) for i in range(119)]
    e += [(200, 200 + i) for i in range(1, 80)]
    e += [(400, 401), (401, 402), (402, 400), (500, 500), (600, 601), (601, 600)]
    edges = torch.tensor(e, dtype=torch.int64, device="cuda")
    tg = cgt.TupleGraph(edges, torch.full((len(e),), 0.5, device="cuda"), len(e))
    return cgt.oned_graph_from_tuple_graph(tg, n), n


def test_msbfs_edge_cases(cgt, oracle):
    """Deep path (119 levels), stars, cycles, self-loops, isolated roots and
    repeated roots; too few depth planes is an error, not a wrong answer,
    and the workspace works again afterwards."""
    h, n = _small_graph(cgt)
    rs, col = _host_csr(h)
    roots = [0, 60, 119, 200, 250, 400, 500, 601, 999, 0, 119]
    ms = cgt.MsBfsState(h, depth_bits=8)
    for mode in (0, 1, 2):
        st = cgt.msbfs_run(h, ms, roots, cgt.MsBfsParams(4.0, mode, 0, 0))
        assert st.error_flags == 0
        d = _depths(cgt, ms)
        for i, r in enumerate(roots):
            _, od = oracle.bfs(rs, col, n, r)
            assert np.array_equal(d[i], od), (mode, r)
    shallow = cgt.MsBfsState(h, depth_bits=3)
    with pytest.raises(ValueError, match="deeper"):
        cgt.msbfs_run(h, shallow, [0])
    st = cgt.msbfs_run(h, shallow, [200, 400, 999])  # depths <= 2: fits 3 planes
    assert st.error_flags == 0
    d = _depths(cgt, shallow)
    for i, r in enumerate([200, 400, 999]):
        _, od = oracle.bfs(rs, col, n, r)
        assert np.array_equal(d[i], od)
    with pytest.raises(ValueError):
        cgt.msbfs_run(h, ms, [])
    with pytest.raises(ValueError):
        cgt.msbfs_run(h, ms, [0] * 257)
    with pytest.raises(ValueError):
        cgt.msbfs_run(h, ms, [n])
