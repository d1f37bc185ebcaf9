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
