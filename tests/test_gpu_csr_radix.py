"""Canonical CSR by LSD radix sort (g5_csr_radix_count + g5_csr_radix_fill):
the same row starts, column and weights as the partition-and-row-sort build
(g5_csr_count + g5_csr_fill_sorted) and as numpy's canonical order, for
Kronecker graphs and for inputs with self-loops only, one vertex, vertex
counts that are not powers of two, long runs of empty rows, and duplicate
runs of every length class (one thread, the block sort, the tiled sort);
bad input is refused with an error, never written out of bounds."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _np(t):
    return t.cpu().numpy()


def _canonical(e: np.ndarray, wt: np.ndarray, n: int):
    """numpy restatement: both directions of every non-loop edge, rows
    sorted by (neighbour, weight bits)."""
    keep = e[:, 0] != e[:, 1]
    e, wt = e[keep], wt[keep]
    src = np.concatenate([e[:, 0], e[:, 1]]).astype(np.int64)
    dst = np.concatenate([e[:, 1], e[:, 0]]).astype(np.int64)
    wb = np.concatenate([wt, wt]).view(np.uint32)
    order = np.lexsort((wb, dst, src))
    rs = np.zeros(n + 1, dtype=np.int64)
    rs[1:] = np.cumsum(np.bincount(src, minlength=n))
    return rs, dst[order].astype(np.uint32), wb[order]


def _radix(cgt, e: torch.Tensor, wt: torch.Tensor, n: int, col64: bool = False):
    """Direct C-ABI build; returns (rc, rowstarts, col, w, col64)."""
    lib = cgt.lib
    m = e.shape[0]
    nb = C.c_uint64()
    assert lib.g5_csr_radix_workspace_size(n, m, C.byref(nb)) == 0
    work = torch.zeros(nb.value, dtype=torch.uint8, device="cuda")
    ne = C.c_uint64()
    rc = lib.g5_csr_radix_count(e.data_ptr() if m else None, m, n, work.data_ptr(), work.numel(), C.byref(ne), None)
    if rc:
        return rc, None, None, None, None
    E = ne.value
    rs = torch.full((n + 1,), -7, dtype=torch.int64, device="cuda")
    col = torch.empty(max(E, 1), dtype=torch.int32, device="cuda")
    w = torch.empty(max(E, 1), dtype=torch.float32, device="cuda")
    c64 = torch.empty(max(E, 1), dtype=torch.int64, device="cuda") if col64 else None
    rc = lib.g5_csr_radix_fill(e.data_ptr() if m else None, wt.data_ptr() if m else None, m, n, E, work.data_ptr(),
                               work.numel(), rs.data_ptr(), col.data_ptr(), w.data_ptr(),
                               c64.data_ptr() if col64 else None, None)
    torch.cuda.synchronize()
    return rc, rs, col[:E], w[:E], None if c64 is None else c64[:E]


@pytest.mark.parametrize("scale,seed", [(12, (2, 3)), (16, (7, 11)), (20, (5, 9))])
def test_radix_equals_partition_build(cgt, scale, seed):
    s = cgt.make_mrg_seed(*seed)
    tg = cgt.generate_kronecker_range(s, scale, 0, 16 << scale)
    kw = dict(with_column64=True, with_main=False, bfs_order=False, sssp_renumber=False)
    a = cgt.oned_graph_from_tuple_graph(tg, 1 << scale, radix=True, **kw)
    b = cgt.oned_graph_from_tuple_graph(tg, 1 << scale, radix=False, **kw)
    assert a.nlocaledges == b.nlocaledges
    for x, y in ((a.rowstarts, b.rowstarts), (a.col, b.col), (a.w, b.w), (a.column, b.column),
                 (a.scol, b.scol), (a.sw, b.sw), (a.light_deg, b.light_deg), (a.tiny_deg, b.tiny_deg)):
        assert torch.equal(x, y)


def test_radix_small_inputs_against_numpy(cgt):
    rng = np.random.default_rng(11)
    cases = []
    # n not a power of two; self-loops and duplicates; vertices 10..899 have no edges
    n = 1000
    lo = rng.integers(0, 10, size=(3000, 2))
    hi = rng.integers(900, 1000, size=(3000, 2))
    e = np.concatenate([lo, hi, np.stack([lo[:, 0], hi[:, 1]], 1)])
    e[::17, 1] = e[::17, 0]  # self-loops
    cases.append((e, n))
    cases.append((np.array([[3, 3], [5, 5]]), 8))                 # self-loops only: no entries
    cases.append((np.array([[0, 0]]), 1))                           # one vertex
    cases.append((np.array([[6, 2]]), 7))                           # one edge
    cases.append((rng.integers(0, 3, size=(20_000, 2)), 3))         # a dense tiny graph, long duplicate runs
    hub = np.stack([np.zeros(70_000, dtype=np.int64), rng.integers(1, 5, size=70_000)], 1)
    cases.append((hub, 1 << 20))                                    # runs beyond 4096 entries, empty tail rows
    for e, n in cases:
        e = e.astype(np.int64)
        wt = rng.random(e.shape[0], dtype=np.float32)
        wt[::5] = wt[0]  # equal weights inside runs too
        rc, rs, col, w, c64 = _radix(cgt, torch.from_numpy(e).cuda(), torch.from_numpy(wt).cuda(), n, col64=True)
        assert rc == 0, cgt.lib.g5_last_error()
        want_rs, want_col, want_w = _canonical(e, wt, n)
        assert np.array_equal(_np(rs), want_rs)
        assert np.array_equal(_np(col).view(np.uint32), want_col)
        assert np.array_equal(_np(w).view(np.uint32), want_w)
        assert np.array_equal(_np(c64), want_col.astype(np.int64))


def test_radix_is_deterministic(cgt):
    s = cgt.make_mrg_seed(3, 4)
    tg = cgt.generate_kronecker_range(s, 18, 0, 16 << 18)
    outs = [_radix(cgt, tg.edges, tg.weights, 1 << 18) for _ in range(2)]
    for x, y in zip(outs[0][1:4], outs[1][1:4]):
        assert torch.equal(x, y)


def test_radix_refuses_bad_input(cgt):
    lib = cgt.lib
    dev = "cuda"
    e = torch.tensor([[0, 1], [1, 9]], dtype=torch.int64, device=dev)  # 9 >= n
    rc, *_ = _radix(cgt, e, torch.ones(2, device=dev), 4)
    assert rc == -1 and b">= nverts" in lib.g5_last_error()
    # edges changed between the count and the fill: same entry count, other rows
    n, m = 4, 3
    nb = C.c_uint64()
    lib.g5_csr_radix_workspace_size(n, m, C.byref(nb))
    work = torch.zeros(nb.value, dtype=torch.uint8, device=dev)
    e1 = torch.tensor([[0, 1], [1, 2], [2, 3]], dtype=torch.int64, device=dev)
    e2 = torch.tensor([[0, 1], [1, 2], [0, 3]], dtype=torch.int64, device=dev)
    wt = torch.ones(m, device=dev)
    ne = C.c_uint64()
    assert lib.g5_csr_radix_count(e1.data_ptr(), m, n, work.data_ptr(), work.numel(), C.byref(ne), None) == 0
    rs = torch.empty(n + 1, dtype=torch.int64, device=dev)
    col = torch.empty(ne.value, dtype=torch.int32, device=dev)
    w = torch.empty(ne.value, dtype=torch.float32, device=dev)
    rc = lib.g5_csr_radix_fill(e2.data_ptr(), wt.data_ptr(), m, n, ne.value, work.data_ptr(), work.numel(),
                               rs.data_ptr(), col.data_ptr(), w.data_ptr(), None, None)
    assert rc == -1 and b"differ" in lib.g5_last_error()
    # a fill whose entry count is not the counted one
    rc = lib.g5_csr_radix_fill(e1.data_ptr(), wt.data_ptr(), m, n, ne.value - 2, work.data_ptr(), work.numel(),
                               rs.data_ptr(), col.data_ptr(), w.data_ptr(), None, None)
    assert rc == -1 and b"g5_csr_radix_count" in lib.g5_last_error()
    # too little scratch
    rc = lib.g5_csr_radix_count(e1.data_ptr(), m, n, work.data_ptr(), 64, C.byref(ne), None)
    assert rc == -2
