"""SSSP under the serving mix: many sources searched at once on several
streams, each on a capped grid (an eighth of the device), with the bucket and
sub-bucket opens checked for vertices queued twice (check_opens: a duplicate
fails the search).  Every status must be OK and every result bit-equal to the
same source searched alone on the full grid, which the oracle pins for some
sources.  Sub-buckets forced on (sub_min=1) and heavy phases forced to pull
stress the queue paths that deferred pushes race on."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NSTREAMS = 4


def _np(t):
    return t.cpu().numpy()


def _graph(cgt, scale):
    return cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), scale, 16 << scale)


def _sources(cgt, g, k_runner, k_random, seed):
    """The runner's first roots plus random vertices of nonzero degree."""
    rs = _np(g.rowstarts)
    deg = rs[1:] - rs[:-1]
    rng = np.random.default_rng(seed)
    cand = np.nonzero(deg > 0)[0]
    extra = rng.choice(cand, size=k_random, replace=False).tolist()
    return cgt.generate_bfs_roots(g, 2, 3, k_runner) + [int(v) for v in extra]


def _alone(cgt, g, roots):
    """Each source alone, full grid, opens checked: (dist bits, pred)."""
    s = cgt.SsspState(g)
    out = {}
    for r in roots:
        cgt.oned_graph_sssp_run(g, s, r, check_opens=True)
        cgt.sssp_status(s)
        out[r] = (_np(s.dist).view(np.uint32).copy(), _np(s.pred).copy())
    return out


def _mix(cgt, g, roots, want, modes):
    """Sources dealt round-robin to NSTREAMS streams, one state each, every
    launch on an eighth of the device; a round launches one search per
    stream before any is checked, so the searches overlap on the GPU."""
    _, max_blocks = cgt.search_grid("sssp", g.nglobalverts)
    blocks = max(1, max_blocks // 8)
    streams = [torch.cuda.Stream() for _ in range(NSTREAMS)]
    states = [cgt.SsspState(g) for _ in range(NSTREAMS)]
    vw = cgt._val_work(g)
    jobs = [(r, m) for r in roots for m in modes]
    checked = 0
    for i in range(0, len(jobs), NSTREAMS):
        batch = list(zip(jobs[i:i + NSTREAMS], streams, states))
        for (r, (pull, sub_min)), st, s in batch:
            cgt.oned_graph_sssp_reset(s, stream=st)
            cgt.oned_graph_sssp_traverse(g, s, r, blocks=blocks, pull=pull, sub_min=sub_min, small=False,
                                         stream=st, check_opens=True)
        for (r, mode), st, s in batch:
            cgt.sssp_status(s, stream=st)  # raises on any device error (capacity, duplicate, timeout)
            st.synchronize()
            d, p = want[r]
            assert np.array_equal(_np(s.dist).view(np.uint32), d), (r, mode)
            assert np.array_equal(_np(s.pred), p), (r, mode)
            assert cgt.sssp_validate(g, r, s.dist, s.pred, vw) == 0, (r, mode)
            checked += 1
    torch.cuda.synchronize()
    return checked


MODES = ((0.0, 0), (0.0, 1), (1e-9, 1), (-1.0, -1))


def test_sssp_mix_scale22_against_alone_and_oracle(cgt, oracle):
    g = _graph(cgt, 22)
    roots = _sources(cgt, g, 8, 8, seed=22)
    want = _alone(cgt, g, roots)
    rs, col, w = _np(g.rowstarts).view(np.uint64), _np(g.col).view(np.uint32), _np(g.w)
    for r in roots[:2]:
        od, _ = oracle.sssp(rs, col, w, g.nglobalverts, r)
        assert np.array_equal(want[r][0], od.view(np.uint32)), r
    assert _mix(cgt, g, roots, want, MODES) == len(roots) * len(MODES)


def test_sssp_mix_scale24_against_alone(cgt):
    g = _graph(cgt, 24)
    roots = _sources(cgt, g, 4, 4, seed=24)
    want = _alone(cgt, g, roots)
    assert _mix(cgt, g, roots, want, MODES[:2]) == len(roots) * 2


@pytest.mark.parametrize("delta", [0.1, 0.05, 0.25])
def test_sssp_checked_opens_small_graph_dense_buckets(cgt, oracle, delta):
    """SCALE 16 with every bucket split into sub-buckets and grids from one
    block to the whole device: no queue ever holds a vertex twice, and the
    distances equal the oracle's."""
    g = _graph(cgt, 16)
    rs, col, w = _np(g.rowstarts).view(np.uint64), _np(g.col).view(np.uint32), _np(g.w)
    s = cgt.SsspState(g)
    _, max_blocks = cgt.search_grid("sssp", g.nglobalverts)
    for r in cgt.generate_bfs_roots(g, 2, 3, 4):
        od, _ = oracle.sssp(rs, col, w, g.nglobalverts, r)
        for blocks in (1, 7, max_blocks // 8, 0):
            for pull, sub_min in ((0.0, 1), (1e-9, 1), (0.0, 0)):
                cgt.oned_graph_sssp_run(g, s, r, delta=delta, blocks=blocks, pull=pull, sub_min=sub_min,
                                        small=False, check_opens=True)
                cgt.sssp_status(s)
                assert np.array_equal(_np(s.dist).view(np.uint32), od.view(np.uint32)), (r, blocks, pull, sub_min)


def test_renumbered_copy_same_distances(cgt, oracle):
    """The SSSP on its degree-renumbered copy (the default) and on the split
    copy in the caller's numbering give bit-identical distances and valid
    parents, for main-component and small-component roots, with and without
    pre-filled outputs; the copy holds each row's entries renamed, in order;
    perm and inv are inverse permutations; perm without inv is refused."""
    scale = 16
    g = cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), scale, 16 << scale)
    assert g.sr is not None
    n = g.nglobalverts
    perm, inv = _np(g.sr.perm).astype(np.int64), _np(g.sr.inv).astype(np.int64)
    assert np.array_equal(perm[inv], np.arange(n)) and np.array_equal(np.sort(perm), np.arange(n))
    deg = np.diff(_np(g.rowstarts))
    assert (np.diff(deg[inv]) <= 0).all()  # decreasing degree
    rs, rs2 = _np(g.rowstarts), _np(g.sr.rowstarts)
    scol, scol2 = _np(g.scol).astype(np.int64), _np(g.sr.col).astype(np.int64)
    for i in (0, 1, 2, n // 2, n - 1):
        o = inv[i]
        assert np.array_equal(perm[scol[rs[o]:rs[o + 1]]], scol2[rs2[i]:rs2[i + 1]])
        assert _np(g.sr.light_deg)[i] == _np(g.light_deg)[o] and _np(g.sr.tiny_deg)[i] == _np(g.tiny_deg)[o]
    roots = cgt.generate_bfs_roots(g, 2, 3, 64)
    small = [r for r in roots if not g.in_main_component(r)]
    plain = cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), scale, 16 << scale, sssp_renumber=False)
    a, b, vw = cgt.SsspState(g), cgt.SsspState(plain), cgt._val_work(g)
    for r in roots[:4] + small[:2]:
        for prefill in (True, False):
            if prefill:
                cgt.oned_graph_sssp_run(g, a, r)
            else:
                cgt.oned_graph_sssp_reset(a)
                cgt.lib.g5_sssp_reset(n, None, None, cgt._ptr(a.work), a.work.numel(), None)
                a.was_reset = True
                cgt.oned_graph_sssp_traverse(g, a, r)
            cgt.sssp_status(a)
            cgt.oned_graph_sssp_run(plain, b, r)
            assert torch.equal(a.dist.view(torch.int32), b.dist.view(torch.int32)), (r, prefill)
            assert cgt.sssp_validate(g, r, a.dist, a.pred, vw) == 0, (r, prefill)  # on the renumbered copy
            assert cgt.sssp_validate(plain, r, a.dist, a.pred, vw) == 0, (r, prefill)  # in the caller's numbering
    # planted mistakes: both validators count the same errors
    bad = a.dist.clone()
    bad[torch.nonzero(bad > 0)[:5, 0]] *= 1.25
    assert cgt.sssp_validate(g, roots[0], bad, a.pred, vw) == cgt.sssp_validate(plain, roots[0], bad, a.pred, vw) > 0
    bfs = cgt.BfsState(g)
    cgt.oned_graph_bfs_run(g, bfs, roots[0])
    d = cgt.bfs_compute_dist_from_pred(g, bfs, roots[0])
    assert cgt.bfs_validate(g, roots[0], bfs.pred, d, vw) == cgt.bfs_validate(plain, roots[0], bfs.pred, d, vw) == 0
    badp = bfs.pred.clone()
    reached = torch.nonzero(badp >= 0)[:, 0]
    badp[reached[1:6]] = reached[10:15]
    badp[reached[6]] = n + 7
    assert cgt.bfs_validate(g, roots[0], badp, d, vw) == cgt.bfs_validate(plain, roots[0], badp, d, vw) > 0
    # the one-block search on the renumbered copy (the Python API runs small
    # components on the caller-numbered copy; the C ABI and the reference
    # API can run them on either)
    for r in small[:2]:
        cgt.oned_graph_sssp_run(plain, b, r)
        for rep in range(2):  # the second reset undoes only this search's vertices
            cgt.oned_graph_sssp_reset(a)
            ps = cgt.SsspParams(0.1, 1, 0.0, 0, 1, cgt._ptr(g.sr.tiny_deg), 0, 0, 0, cgt._ptr(g.sr.perm),
                                cgt._ptr(g.sr.inv))
            assert cgt.lib.g5_sssp_traverse(cgt._ptr(g.sr.rowstarts), cgt._ptr(g.sr.col), cgt._ptr(g.sr.w),
                                            cgt._ptr(g.sr.light_deg), g.light_delta, n, int(r), cgt._ptr(a.dist),
                                            cgt._ptr(a.pred), cgt._ptr(a.work), a.work.numel(), cgt.C.byref(ps),
                                            None) == 0
            cgt.sssp_status(a)
            assert torch.equal(a.dist.view(torch.int32), b.dist.view(torch.int32)), (r, rep)
            assert cgt.sssp_validate(g, r, a.dist, a.pred, vw) == 0, (r, rep)
    p = cgt.SsspParams(0.1, 0, 0.0, 0, 0, None, 0, 0, 0, cgt._ptr(g.sr.perm), None)
    rc = cgt.lib.g5_sssp_traverse(cgt._ptr(g.sr.rowstarts), cgt._ptr(g.sr.col), cgt._ptr(g.sr.w), cgt._ptr(g.sr.light_deg),
                                  g.light_delta, n, int(roots[0]), cgt._ptr(a.dist), cgt._ptr(a.pred), cgt._ptr(a.work),
                                  a.work.numel(), cgt.C.byref(p), None)
    assert rc == -1 and b"perm and inv" in cgt.lib.g5_last_error()
