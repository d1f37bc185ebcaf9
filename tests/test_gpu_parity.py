"""CUDA path (libg500b through its C ABI) against the reference fixtures and
the CPU oracle.  Integer/index outputs are compared bit for bit; the float32
SSSP distances are compared bit for bit as well (tolerance 0: the float
fixed point is unique, see oracle/g500_oracle.c orc_sssp)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from tests.golden.make_golden import golden_hashes, sha

pytestmark = pytest.mark.gpu

INT64_MAX = np.iinfo(np.int64).max


def _np(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def graphs(cgt, oracle):
    """Device graph + oracle CSR per scale."""
    out = {}
    for scale in (12, 14, 16):
        n, m = 1 << scale, 16 << scale
        seed = cgt.make_mrg_seed(2, 3)
        tg = cgt.generate_kronecker_range(seed, scale, 0, m)
        g = cgt.oned_graph_from_tuple_graph(tg, n, with_column64=True)
        oe, ow = oracle.generate_kronecker_range(np.array(seed, np.uint32), scale, 0, m)
        ors, ocol, ocw = oracle.csr_build(oe, ow, n)
        out[scale] = dict(tg=tg, g=g, n=n, oe=oe, ow=ow, ors=ors, ocol=ocol, ocw=ocw)
    return out


def test_generator_bit_exact(graphs, golden_dump):
    d = graphs[golden_dump["scale"]]
    e = _np(d["tg"].edges).view(np.uint64)
    w = _np(d["tg"].weights)
    assert e[:16].tolist() == golden_dump["first_edges"]
    assert sha(e) == golden_dump["edges_sha256"]
    assert sha(w) == golden_dump["weights_sha256"]


def test_generator_matches_oracle_and_ranges(cgt, graphs):
    d = graphs[16]
    assert np.array_equal(_np(d["tg"].edges).view(np.uint64), d["oe"])
    assert np.array_equal(_np(d["tg"].weights).view(np.uint32), d["ow"].view(np.uint32))
    seed = cgt.make_mrg_seed(2, 3)
    for start, end in [(0, 1), (1, 2), (777, 778), (12345, 54321), (2**20 - 3, 2**20)]:
        sub = cgt.generate_kronecker_range(seed, 16, start, end)
        assert np.array_equal(_np(sub.edges).view(np.uint64), d["oe"][start:end]), (start, end)
        assert np.array_equal(_np(sub.weights).view(np.uint32), d["ow"][start:end].view(np.uint32))
    empty = cgt.generate_kronecker_range(seed, 16, 10, 10)
    assert empty.edges_size == 0


def test_generator_other_seeds_and_scales(cgt, oracle):
    for s1, s2, scale in [(1, 1, 1), (12345, 67890, 9), (2**63 + 5, 7, 20)]:
        seed = cgt.make_mrg_seed(s1, s2)
        m = min(16 << scale, 1 << 18)
        tg = cgt.generate_kronecker_range(seed, scale, 3, m)
        oe, ow = oracle.generate_kronecker_range(np.array(seed, np.uint32), scale, 3, m)
        assert np.array_equal(_np(tg.edges).view(np.uint64), oe)
        assert np.array_equal(_np(tg.weights).view(np.uint32), ow.view(np.uint32))


def test_csr_matches_reference(graphs, golden_dump):
    d = graphs[golden_dump["scale"]]
    g = d["g"]
    h = golden_hashes(_np(d["tg"].edges).view(np.uint64), _np(d["tg"].weights),
                      _np(g.rowstarts).view(np.uint64), _np(g.col), _np(g.w))
    for k in ("rowstarts_sha256", "csr_canonical_sha256"):
        assert h[k] == golden_dump[k]
    assert g.nlocaledges == golden_dump["nentries"]
    assert np.array_equal(_np(g.column), _np(g.col).astype(np.int64))


def test_csr_light_partition(graphs):
    g = graphs[16]["g"]
    rs = _np(g.rowstarts)
    w = _np(g.sssp_w)
    ld = _np(g.light_deg).astype(np.int64)
    src = np.repeat(np.arange(g.nglobalverts), np.diff(rs))
    pos = np.arange(rs[-1]) - rs[src]
    assert np.array_equal(pos < ld[src], w < np.float32(0.1))


def test_csr_tiny_split(cgt, graphs):
    """g5_csr_split_tiny: every row's light part starts with its entries
    below light_delta / 30 (tiny_deg of them), the other light entries after
    them; the rows' multisets stay those of the fill (the canonical-row hash
    test covers them) and a second split changes nothing."""
    for scale in (12, 16):
        g = graphs[scale]["g"]
        rs = _np(g.rowstarts)
        w = _np(g.sssp_w)
        ld = _np(g.light_deg).astype(np.int64)
        td = _np(g.tiny_deg).astype(np.int64)
        src = np.repeat(np.arange(g.nglobalverts), np.diff(rs))
        pos = np.arange(rs[-1]) - rs[src]
        tiny = np.float32(g.light_delta) / np.float32(30)
        assert np.array_equal(pos < td[src], (pos < ld[src]) & (w < tiny))
        assert td.sum() > 0 and np.all(td <= ld)
        assert np.array_equal(_np(g.column), _np(g.col).astype(np.int64))
        col, ww = _np(g.sssp_col).copy(), w.copy()
        td2 = cgt._split_tiny(g.rowstarts, g.sssp_col, g.sssp_w, None, g.light_deg, g.nglobalverts, g.light_delta,
                              None)
        assert np.array_equal(_np(td2), td)
        assert np.array_equal(_np(g.sssp_col), col) and np.array_equal(_np(g.sssp_w), ww)


def test_csr_edge_cases(cgt):
    dev = "cuda"
    # only self loops -> no entries, every vertex isolated
    edges = torch.tensor([[1, 1], [2, 2], [3, 3]], dtype=torch.int64, device=dev)
    tg = cgt.TupleGraph(edges, torch.ones(3, device=dev), 3)
    g = cgt.oned_graph_from_tuple_graph(tg, 8)
    assert g.nlocaledges == 0 and _np(g.rowstarts).tolist() == [0] * 9
    # empty edge list
    tg = cgt.TupleGraph(torch.empty((0, 2), dtype=torch.int64, device=dev), torch.empty(0, device=dev), 0)
    g = cgt.oned_graph_from_tuple_graph(tg, 4)
    assert g.nlocaledges == 0
    # duplicates are kept, both directions
    edges = torch.tensor([[0, 1], [1, 0], [0, 1], [2, 3]], dtype=torch.int64, device=dev)
    tg = cgt.TupleGraph(edges, torch.tensor([0.5, 0.05, 0.5, 1.0], device=dev), 4)
    g = cgt.oned_graph_from_tuple_graph(tg, 4)
    assert _np(g.rowstarts).tolist() == [0, 3, 6, 7, 8]
    assert sorted(_np(g.col)[0:3].tolist()) == [1, 1, 1]
    assert _np(g.light_deg).tolist() == [1, 1, 0, 0]
    # an endpoint outside [0, N) is rejected
    edges = torch.tensor([[0, 9]], dtype=torch.int64, device=dev)
    tg = cgt.TupleGraph(edges, torch.ones(1, device=dev), 1)
    with pytest.raises(ValueError):
        cgt.oned_graph_from_tuple_graph(tg, 4)


def test_roots_match_reference(cgt, graphs, golden_dump):
    g = graphs[golden_dump["scale"]]["g"]
    assert cgt.generate_bfs_roots(g, 2, 3, len(golden_dump["roots"])) == golden_dump["roots"]


def test_bfs_depth_matches_reference(cgt, graphs, golden_dump):
    """Depth bit-exact with the reference's (bfs_compute_dist_from_pred over
    its BFS) for every fixture root; our parent tree validates and gives the
    reference's TEPS edge count."""
    d = graphs[golden_dump["scale"]]
    g = d["g"]
    bfs = cgt.BfsState(g)
    vw = cgt._val_work(g)
    for pr in golden_dump["per_root"]:
        r = pr["root"]
        cgt.oned_graph_bfs_run(g, bfs, r)
        depth = _np(bfs.depth).astype(np.int64)
        assert sha(depth) == pr["depth_sha256"], r
        dist = cgt.bfs_compute_dist_from_pred(g, bfs, r)
        assert sha(_np(dist)) == pr["depth_sha256"], r
        assert cgt.bfs_validate(g, r, bfs.pred, dist, vw) == 0
        assert cgt.edge_count(g, bfs.pred, vw) == pr["nedge"]
        st = cgt.bfs_stats(bfs)
        assert st.reached == pr["reached"]


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("blocks", [0, 1, 3])
def test_bfs_modes_and_grids_agree(cgt, oracle, graphs, mode, blocks):
    """Direction-optimizing, top-down-only and bottom-up-only BFS on any
    grid size give the oracle's depth array and a valid tree."""
    d = graphs[16]
    g = d["g"]
    bfs = cgt.BfsState(g)
    roots = cgt.generate_bfs_roots(g, 2, 3, 4)
    params = cgt.BfsParams(14.0, 24.0, mode, blocks)
    for r in roots:
        cgt.oned_graph_bfs_run(g, bfs, r, params)
        _, odepth = oracle.bfs(d["ors"], d["ocol"], d["n"], r)
        assert np.array_equal(_np(bfs.depth).astype(np.int64), odepth)
        pred = _np(bfs.pred)
        dist = oracle.bfs_dist_from_pred(d["ors"], d["ocol"], d["n"], pred, r)
        assert oracle.bfs_validate(d["ors"], d["ocol"], d["n"], r, pred, dist) == 0


def test_bfs_isolated_root_and_bad_root(cgt, graphs):
    g = graphs[12]["g"]
    rs = _np(g.rowstarts)
    iso = int(np.nonzero(np.diff(rs) == 0)[0][0])
    bfs = cgt.BfsState(g)
    cgt.oned_graph_bfs_run(g, bfs, iso)
    pred = _np(bfs.pred)
    assert pred[iso] == iso and (pred != -1).sum() == 1
    assert cgt.bfs_stats(bfs).reached == 1
    with pytest.raises(ValueError):
        cgt.oned_graph_bfs_run(g, bfs, g.nglobalverts)


def _corruptions(pred, n, root, rng):
    reached = np.nonzero((pred != -1) & (np.arange(n) != root))[0]
    out = []
    a = pred.copy()
    a[reached[:5]] = reached[10:15]
    out.append(a)
    b = pred.copy()
    b[reached[0]] = n + 7
    b[reached[1]] = -5
    out.append(b)
    c = pred.copy()
    c[root] = reached[0]
    out.append(c)
    dd = pred.copy()
    dd[reached[2]] = reached[3]
    dd[reached[3]] = reached[2]  # a two-cycle
    out.append(dd)
    e = pred.copy()
    e[rng.choice(np.nonzero(pred == -1)[0], 3)] = root
    out.append(e)
    return out


def test_validation_counts_match_oracle(cgt, oracle, graphs):
    """Planted mistakes (on the CPU, in the inputs): the GPU's
    bfs_compute_dist_from_pred, seven-rule validator and edge count give the
    oracle's arrays and counts."""
    d = graphs[12]
    g, n = d["g"], d["n"]
    bfs = cgt.BfsState(g)
    vw = cgt._val_work(g)
    rng = np.random.default_rng(5)
    for r in cgt.generate_bfs_roots(g, 2, 3, 3):
        cgt.oned_graph_bfs_run(g, bfs, r)
        pred = _np(bfs.pred)
        for bad in _corruptions(pred, n, r, rng):
            bfs.pred.copy_(torch.from_numpy(bad))
            dist = _np(cgt.bfs_compute_dist_from_pred(g, bfs, r))
            odist = oracle.bfs_dist_from_pred(d["ors"], d["ocol"], n, bad, r)
            assert np.array_equal(dist, odist)
            got = cgt.bfs_validate(g, r, bfs.pred, bfs.dist, vw)
            assert got == oracle.bfs_validate(d["ors"], d["ocol"], n, r, bad, odist) and got > 0
            assert cgt.edge_count(g, bfs.pred, vw) == oracle.edge_count(d["ors"], d["ocol"], n, bad)
        cgt.oned_graph_bfs_run(g, bfs, r)
        good = cgt.bfs_compute_dist_from_pred(g, bfs, r)
        skew = _np(good).copy()
        skew[np.nonzero(skew > 0)[0][:4]] += 2
        want = oracle.bfs_validate(d["ors"], d["ocol"], n, r, _np(bfs.pred), skew)
        assert cgt.bfs_validate(g, r, bfs.pred, torch.from_numpy(skew).cuda(), vw) == want > 0


def test_sssp_matches_reference(cgt, graphs, golden_dump):
    d = graphs[golden_dump["scale"]]
    g = d["g"]
    s = cgt.SsspState(g)
    vw = cgt._val_work(g)
    for pr in golden_dump["per_root"]:
        r = pr["root"]
        cgt.oned_graph_sssp_run(g, s, r)
        cgt.sssp_status(s)
        assert sha(_np(s.dist)) == pr["sssp_dist_sha256"], r
        assert cgt.sssp_validate(g, r, s.dist, s.pred, vw) == 0
        assert cgt.edge_count(g, s.pred, vw) == pr["nedge"]


@pytest.mark.parametrize("delta", [0.1, 0.07, 0.04, 0.25, 1.0, 4.0])
def test_sssp_any_delta_same_bits(cgt, oracle, graphs, delta):
    """The distances do not depend on delta (the CSR's light/heavy split at
    0.1 used for every delta up to 0.1, weight filtering above)."""
    d = graphs[16]
    g = d["g"]
    s = cgt.SsspState(g)
    for r in cgt.generate_bfs_roots(g, 2, 3, 3):
        cgt.oned_graph_sssp_run(g, s, r, delta=delta)
        cgt.sssp_status(s)
        od, _ = oracle.sssp(d["ors"], d["ocol"], d["ocw"], d["n"], r)
        assert np.array_equal(_np(s.dist).view(np.uint32), od.view(np.uint32))
        assert oracle.sssp_validate(d["ors"], d["ocol"], d["ocw"], d["n"], r, _np(s.dist), _np(s.pred)) == 0


@pytest.mark.parametrize("delta", [0.1, 0.25, 0.05])
def test_sssp_pull_push_and_sub_buckets_same_bits(cgt, oracle, graphs, delta):
    """Heavy phases run as pulls (every unsettled vertex scans its own heavy
    entries) and buckets split into sub-buckets give the same distances as
    the oracle and the same parents as plain push-only buckets: the parent is
    the smallest u on a tight edge either way.  pull=1e-9 pulls whenever a
    bucket has rows, -1 never; sub_min=1 splits every bucket with a light
    frontier, -1 never.  Inside a sub-bucket the relaxations that leave it
    wait for its settle pass."""
    d = graphs[16]
    g = d["g"]
    s = cgt.SsspState(g)
    for r in cgt.generate_bfs_roots(g, 2, 3, 3):
        cgt.oned_graph_sssp_run(g, s, r, delta=delta, pull=-1.0, sub_min=-1)
        tr = cgt.sssp_trace(s)
        assert tr["counts"]["pulls"] == 0 and 5 not in tr["kind"]
        push_pred = _np(s.pred).copy()
        od, _ = oracle.sssp(d["ors"], d["ocol"], d["ocw"], d["n"], r)
        for pull, sub_min in ((1e-9, -1), (-1.0, 1), (1e-9, 1), (0.0, 0), (4.0, 64)):
            cgt.oned_graph_sssp_run(g, s, r, delta=delta, pull=pull, sub_min=sub_min, small=False)
            tr = cgt.sssp_trace(s)
            if pull == 1e-9:
                assert tr["counts"]["pulls"] > 0
            if sub_min == 1:
                # split (5), sub-buckets opened (4), deferred edges settled (6)
                assert 5 in tr["kind"] and 4 in tr["kind"] and 6 in tr["kind"]
            assert np.array_equal(_np(s.dist).view(np.uint32), od.view(np.uint32)), (r, pull, sub_min)
            assert np.array_equal(_np(s.pred), push_pred), (r, pull, sub_min)


def test_sssp_small_component_search_same_bits(cgt, oracle, graphs):
    """The lean one-block search (label-correcting rounds, meant for roots
    outside the main component) gives the oracle's distances and the bucketed
    search's parents, from main-component roots too, with outputs pre-filled
    by the reset and with outputs left to the search."""
    d = graphs[16]  # 12 vertices of non-zero degree lie outside its main component
    g = d["g"]
    s = cgt.SsspState(g)
    rs = _np(g.rowstarts)
    small_roots = [v for v in range(d["n"]) if not g.in_main_component(v) and rs[v + 1] > rs[v]][:3]
    assert small_roots
    for r in cgt.generate_bfs_roots(g, 2, 3, 2) + small_roots:
        cgt.oned_graph_sssp_run(g, s, r, small=False)
        want_pred = _np(s.pred).copy()
        od, _ = oracle.sssp(d["ors"], d["ocol"], d["ocw"], d["n"], r)
        for prefill in (True, False):
            if prefill:
                cgt.oned_graph_sssp_reset(s)
            else:  # workspace only: the search writes all N outputs itself
                s.dist.fill_(7.0)
                s.pred.fill_(7)
                assert cgt.lib.g5_sssp_reset(s.max_nlocalverts, None, None, s.work.data_ptr(), s.work.numel(),
                                             None) == 0
            cgt.oned_graph_sssp_traverse(g, s, r, small=True)
            cgt.sssp_status(s)
            assert np.array_equal(_np(s.dist).view(np.uint32), od.view(np.uint32)), (r, prefill)
            assert np.array_equal(_np(s.pred), want_pred), (r, prefill)


def test_sssp_validation_counts_match_oracle(cgt, oracle, graphs):
    d = graphs[12]
    g, n = d["g"], d["n"]
    s = cgt.SsspState(g)
    vw = cgt._val_work(g)
    r = cgt.generate_bfs_roots(g, 2, 3, 1)[0]
    cgt.oned_graph_sssp_run(g, s, r)
    dist, pred = _np(s.dist), _np(s.pred)
    reached = np.nonzero((pred != -1) & (np.arange(n) != r))[0]
    cases = []
    a = dist.copy(); a[reached[:3]] += np.float32(0.125); cases.append((a, pred))
    b = pred.copy(); b[reached[4]] = reached[40]; cases.append((dist, b))
    c = dist.copy(); c[reached[5]] = -1.0; cases.append((c, pred))
    e = dist.copy(); e[r] = 0.5; cases.append((e, pred))
    for cd, cp in cases:
        want = oracle.sssp_validate(d["ors"], d["ocol"], d["ocw"], n, r, cd, cp)
        got = cgt.sssp_validate(g, r, torch.from_numpy(cd).cuda(), torch.from_numpy(cp).cuda(), vw)
        assert got == want > 0


def test_property_checks_scale20(cgt, oracle):
    """Size-independent properties at a larger scale: every BFS tree and SSSP
    result validates, depths equal the oracle's, both directions agree."""
    scale = 20
    n = 1 << scale
    seed = cgt.make_mrg_seed(2, 3)
    tg = cgt.generate_kronecker_range(seed, scale, 0, 16 << scale)
    g = cgt.oned_graph_from_tuple_graph(tg, n)
    rs, col, w = _np(g.rowstarts).view(np.uint64), _np(g.col).view(np.uint32), _np(g.w)
    bfs, s, vw = cgt.BfsState(g), cgt.SsspState(g), cgt._val_work(g)
    for r in cgt.generate_bfs_roots(g, 2, 3, 3):
        cgt.oned_graph_bfs_run(g, bfs, r)
        dist = cgt.bfs_compute_dist_from_pred(g, bfs, r)
        assert cgt.bfs_validate(g, r, bfs.pred, dist, vw) == 0
        _, od = oracle.bfs(rs, col, n, r)
        assert np.array_equal(_np(bfs.depth).astype(np.int64), od)
        cgt.oned_graph_sssp_run(g, s, r)
        cgt.sssp_status(s)
        assert cgt.sssp_validate(g, r, s.dist, s.pred, vw) == 0
        sd, _ = oracle.sssp(rs, col, w, n, r)
        assert np.array_equal(_np(s.dist).view(np.uint32), sd.view(np.uint32))


def test_bounded_wait_reports_timeout_and_context_survives(cgt):
    with pytest.raises(TimeoutError):
        cgt.selftest_wait_timeout(50)
    x = torch.arange(10, device="cuda")
    assert int(x.sum()) == 45


def test_bfs_query_path_and_small_components(cgt, oracle, graphs):
    """g5_bfs_query (pinned root in, stats out) gives the oracle's trees;
    roots outside the main component run on one block with the same result."""
    d = graphs[14]
    g = d["g"]
    bfs = cgt.BfsState(g)
    for r in cgt.generate_bfs_roots(g, 2, 3, 8):
        assert g.in_main_component(r)
        cgt.oned_graph_bfs_reset(bfs, g=g)
        st = cgt.oned_graph_bfs_query(g, bfs, r, with_depth=True)
        _, od = oracle.bfs(d["ors"], d["ocol"], d["n"], r)
        assert np.array_equal(_np(bfs.depth).astype(np.int64), od)
        assert st.reached == int((od != -1).sum()) and st.error_flags == 0
    # A graph with a 300-vertex star-and-chain component and small ones.
    n = 1024
    e = [(0, i) for i in range(1, 200)] + [(i, i + 1) for i in range(199, 299)]
    e += [(500, 501), (600, 601), (601, 602), (602, 603), (700, 700)]
    edges = torch.tensor(e, dtype=torch.int64, device="cuda")
    tg = cgt.TupleGraph(edges, torch.full((len(e),), 0.5, device="cuda"), len(e))
    h = cgt.oned_graph_from_tuple_graph(tg, n)
    assert h.in_main_component(0) and h.in_main_component(299)
    assert not h.in_main_component(500) and not h.in_main_component(603) and not h.in_main_component(700)
    rs, col = _np(h.rowstarts).view(np.uint64), _np(h.col).view(np.uint32)
    hb = cgt.BfsState(h)
    for r in (0, 250, 500, 601, 603, 700, 1000):
        cgt.oned_graph_bfs_reset(hb, g=h)
        st = cgt.oned_graph_bfs_query(h, hb, r, with_depth=True)
        _, od = oracle.bfs(rs, col, n, r)
        assert np.array_equal(_np(hb.depth).astype(np.int64), od), r
        assert st.reached == int((od != -1).sum())
        if not h.in_main_component(r):
            assert st.solo_levels == st.levels  # the whole search ran on one block


def test_fused_generator_csr_matches(cgt, graphs, golden_dump):
    """The generator fused into the CSR passes (no edge list) builds the
    reference's CSR: same rowstarts and canonical rows as the fixtures."""
    scale = golden_dump["scale"]
    g = cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), scale, 16 << scale, with_column64=True)
    d = graphs[scale]
    h = golden_hashes(_np(d["tg"].edges).view(np.uint64), _np(d["tg"].weights),
                      _np(g.rowstarts).view(np.uint64), _np(g.col), _np(g.w))
    assert h["rowstarts_sha256"] == golden_dump["rowstarts_sha256"]
    assert h["csr_canonical_sha256"] == golden_dump["csr_canonical_sha256"]
    assert np.array_equal(_np(g.column), _np(g.col).astype(np.int64))
    ref = d["g"]
    assert np.array_equal(_np(g.light_deg), _np(ref.light_deg))
    assert np.array_equal(g.main_bits, ref.main_bits)


def test_sssp_delta_too_small_is_an_error(cgt, graphs):
    """A delta so small that a weight spans more buckets than the ring holds
    is reported (ValueError), not answered wrongly; the next search works."""
    g = graphs[12]["g"]
    ss = cgt.SsspState(g)
    r = cgt.generate_bfs_roots(g, 2, 3, 1)[0]
    with pytest.raises(ValueError, match="larger delta"):
        cgt.oned_graph_sssp_run(g, ss, r, delta=0.01)
        cgt.sssp_status(ss)
    cgt.oned_graph_sssp_run(g, ss, r)
    assert cgt.sssp_status(ss)[0] > 0


@pytest.mark.parametrize("shape", ["dense", "sparse_runs"])
def test_validation_tile_table_edge_cases(cgt, oracle, shape):
    """The validators and the edge count find each entry's row from a
    per-tile table (built by a pre-pass) or, for graphs denser than the
    table allows, by searching rowptr; tiles whose span includes long runs
    of empty rows fall back to a per-entry search.  Every path gives the
    oracle's counts, with and without planted mistakes."""
    rng = np.random.default_rng(11)
    if shape == "dense":  # 400 entries per vertex on average: more tiles than the table holds
        n = 96
        e = rng.integers(0, 64, size=(19_200, 2))  # vertices 64..95 stay unreached
    else:  # a few busy vertices separated by thousands of isolated ones
        n = 1 << 16
        busy = rng.choice(n, 40, replace=False)
        e = np.stack([rng.choice(busy, 60_000), rng.choice(busy, 60_000)], 1)
    e = e[e[:, 0] != e[:, 1]].astype(np.int64)
    wt = rng.random(e.shape[0], dtype=np.float32)
    tg = cgt.TupleGraph(torch.from_numpy(e).cuda(), torch.from_numpy(wt).cuda(), e.shape[0])
    g = cgt.oned_graph_from_tuple_graph(tg, n)
    ors, ocol, ocw = _np(g.rowstarts).view(np.uint64), _np(g.col), _np(g.w)
    vw = cgt._val_work(g)
    bfs, s = cgt.BfsState(g), cgt.SsspState(g)
    r = int(e[0, 0])
    cgt.oned_graph_bfs_run(g, bfs, r)
    dist = cgt.bfs_compute_dist_from_pred(g, bfs, r)
    pred = _np(bfs.pred)
    assert cgt.bfs_validate(g, r, bfs.pred, dist, vw) == 0
    assert cgt.edge_count(g, bfs.pred, vw) == oracle.edge_count(ors, ocol, n, pred) > 0
    for bad in _corruptions(pred, n, r, rng):
        bfs.pred.copy_(torch.from_numpy(bad))
        odist = oracle.bfs_dist_from_pred(ors, ocol, n, bad, r)
        gd = cgt.bfs_compute_dist_from_pred(g, bfs, r)
        assert np.array_equal(_np(gd), odist)
        assert cgt.bfs_validate(g, r, bfs.pred, gd, vw) == oracle.bfs_validate(ors, ocol, n, r, bad, odist)
        assert cgt.edge_count(g, bfs.pred, vw) == oracle.edge_count(ors, ocol, n, bad)
    cgt.oned_graph_sssp_run(g, s, r)
    assert cgt.sssp_validate(g, r, s.dist, s.pred, vw) == 0
    cd = _np(s.dist).copy()
    cd[np.nonzero(cd > 0)[0][:3]] *= np.float32(1.5)
    cp = _np(s.pred)
    want = oracle.sssp_validate(ors, ocol, ocw, n, r, cd, cp)
    assert cgt.sssp_validate(g, r, torch.from_numpy(cd).cuda(), s.pred, vw) == want > 0
