"""g5_bfs_run_static: the BFS for callers that must not allocate device
memory (their memory belongs to another allocator, or they cannot stall on
the device-wide synchronisation cudaMalloc/cudaFree imply).  Its scratch is a
fixed array inside the library, so the call takes only the graph and the
outputs.  Checked through the C ABI against g5_bfs_run (the workspace entry
point): identical depth arrays and reached counts, valid parent trees, on two
calls in a row; oversized graphs are refused.

This file sorts last so that a run stopping at its first failure has already
run every other test; it builds its own graph and runs alone as well."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from tests.conftest import load_package

pytestmark = pytest.mark.gpu


def _static_fn(lib):
    fn = lib.g5_bfs_run_static
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return fn


def test_static_bfs_matches_workspace_bfs():
    G = load_package()
    lib = G.lib
    static_bfs = _static_fn(lib)
    scale = 16
    n = 1 << scale
    tg = G.generate_kronecker_range(G.make_mrg_seed(2, 3), scale, 0, 16 << scale)
    g = G.oned_graph_from_tuple_graph(tg, n)
    roots = G.generate_bfs_roots(g, 2, 3, 2)
    ref = G.BfsState(g)
    pred = torch.empty(n, dtype=torch.int64, device="cuda")
    depth = torch.empty(n, dtype=torch.int32, device="cuda")
    vw = G._val_work(g)
    for r in roots:  # two calls in a row on the shared static scratch
        G.oned_graph_bfs_run(g, ref, r)
        rc = static_bfs(g.rowstarts.data_ptr(), g.col.data_ptr(), n, r, pred.data_ptr(), depth.data_ptr(), None,
                        None)
        assert rc == 0, lib.g5_last_error()
        torch.cuda.synchronize()
        assert torch.equal(depth, ref.depth), r
        assert int((pred != -1).sum()) == int((ref.pred != -1).sum())
        ref.pred.copy_(pred)
        dist = G.bfs_compute_dist_from_pred(g, ref, r)
        assert np.array_equal(dist.cpu().numpy(), depth.cpu().numpy().astype(np.int64))
        assert G.bfs_validate(g, r, pred, dist, vw) == 0


def test_static_bfs_refuses_large_graphs():
    G = load_package()
    static_bfs = _static_fn(G.lib)
    rc = static_bfs(None, None, (1 << 18) + 1, 0, None, None, None, None)
    assert rc == -1 and b"limit" in G.lib.g5_last_error()
