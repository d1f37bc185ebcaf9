"""Autotuner (autotune.py): it times candidates and returns settings that
leave every result unchanged."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g(cgt):
    return cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), 14, 16 << 14)


def test_tuned_settings_keep_results(cgt, g, tmp_path):
    from cgt_b200 import autotune as T
    roots = cgt.generate_bfs_roots(g, 2, 3, 4)
    _, maxb = cgt.search_grid("bfs", g.nglobalverts)
    tb = T.tune_bfs(g, roots, alphas=(10.0, 14.0), betas=(24.0,), grids=(0, maxb),
                    tiles={"chunk": (64, 256), "big_deg": (32, 1024), "lane_entries": (4, 8)})
    # the 4 direction/grid settings, then the defaults' tiles and every other value of each axis
    tiles = {"chunk": (64, 256), "big_deg": (32, 1024), "lane_entries": (4, 8)}
    others = sum(len(set(v) - {T.BFS_DEFAULT_TILES[k]}) for k, v in tiles.items())
    assert tb["candidates"] == 4 + 1 + others and tb["ms"] > 0
    assert tb["chunk"] in (64, 256) and tb["big_deg"] in (32, 1024) and tb["lane_entries"] in (4, 8)
    bfs = cgt.BfsState(g)
    cgt.oned_graph_bfs_run(g, bfs, roots[0])
    want = bfs.depth.clone()
    cgt.oned_graph_bfs_run(g, bfs, roots[0], T.bfs_params(tb))
    assert torch.equal(bfs.depth, want)

    ts = T.tune_sssp(g, roots[:2], deltas=(0.1, 0.3), grids=(0,), tiles={"chunk": (64, 256), "big_deg": (1, 128)})
    ss = cgt.SsspState(g)
    cgt.oned_graph_sssp_run(g, ss, roots[0])
    want = ss.dist.clone()
    cgt.oned_graph_sssp_run(g, ss, roots[0], **T.sssp_kwargs(ts))
    assert torch.equal(ss.dist.view(torch.int32), want.view(torch.int32))

    tm = T.tune_msbfs(g, roots, alphas=(8.0, 32.0), checks=(0, 2))
    ms = cgt.MsBfsState(g)
    cgt.msbfs_run(g, ms, roots, T.msbfs_params(tm))
    d = cgt.msbfs_depths_u8(ms)
    for i, r in enumerate(roots):
        cgt.oned_graph_bfs_run(g, bfs, r)
        got = d[i].to(torch.int32)
        got[got == 255] = -1
        assert torch.equal(got, bfs.depth)

    cache = T.TuningCache(str(tmp_path / "tune.json"))
    first = cache.tuned("sssp", g, roots[:1], deltas=(0.1,), grids=(0,))
    again = T.TuningCache(str(tmp_path / "tune.json")).get("sssp", g)
    assert again == first


@pytest.mark.parametrize("tiles", [dict(big_deg=1, chunk=32, lane_entries=4), dict(big_deg=32, chunk=64),
                                   dict(big_deg=1 << 20, chunk=65536, lane_entries=1024)])
def test_tiles_keep_results(cgt, g, tiles):
    """Every tile setting in range gives the default's BFS depths and SSSP
    distances: the smallest tiles send nearly every list entry through the
    chunked big part, the largest send none."""
    roots = cgt.generate_bfs_roots(g, 2, 3, 3)
    bfs, ss = cgt.BfsState(g), cgt.SsspState(g)
    sssp_tiles = dict(big_deg=tiles["big_deg"], chunk=max(64, tiles["chunk"]))
    for r in roots:
        cgt.oned_graph_bfs_run(g, bfs, r)
        want_depth = bfs.depth.clone()
        p = cgt.BfsParams(14.0, 24.0, 0, 0, tiles["big_deg"], tiles["chunk"], tiles.get("lane_entries", 0))
        cgt.oned_graph_bfs_run(g, bfs, r, p)
        assert torch.equal(bfs.depth, want_depth)
        cgt.oned_graph_sssp_run(g, ss, r)
        want = ss.dist.clone()
        cgt.oned_graph_sssp_run(g, ss, r, **sssp_tiles)
        assert torch.equal(ss.dist.view(torch.int32), want.view(torch.int32))
        cgt.sssp_status(ss)


def test_bad_tiles_rejected(cgt, g):
    bfs, ss = cgt.BfsState(g), cgt.SsspState(g)
    for bad in (dict(chunk=48), dict(chunk=1 << 17), dict(big_deg=-1), dict(lane_entries=6)):
        p = cgt.BfsParams(14.0, 24.0, 0, 0, bad.get("big_deg", 0), bad.get("chunk", 0), bad.get("lane_entries", 0))
        with pytest.raises(cgt.G5InvalidError):
            cgt.oned_graph_bfs_run(g, bfs, 0, p)
    for bad in (dict(chunk=32), dict(chunk=96), dict(big_deg=(1 << 20) + 1)):
        with pytest.raises(cgt.G5InvalidError):
            cgt.oned_graph_sssp_run(g, ss, 0, **bad)
