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
    tb = T.tune_bfs(g, roots, alphas=(10.0, 14.0), betas=(24.0,), grids=(0, maxb))
    assert tb["candidates"] == 4 and tb["ms"] > 0
    bfs = cgt.BfsState(g)
    cgt.oned_graph_bfs_run(g, bfs, roots[0])
    want = bfs.depth.clone()
    cgt.oned_graph_bfs_run(g, bfs, roots[0], T.bfs_params(tb))
    assert torch.equal(bfs.depth, want)

    ts = T.tune_sssp(g, roots[:2], deltas=(0.1, 0.3), grids=(0,))
    ss = cgt.SsspState(g)
    cgt.oned_graph_sssp_run(g, ss, roots[0])
    want = ss.dist.clone()
    cgt.oned_graph_sssp_run(g, ss, roots[0], delta=ts["delta"], blocks=ts["blocks"], pull=ts["pull"],
                            sub_min=ts["sub_min"])
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
