"""Batched SSSP (g5_sssp_multi_run): up to 32 sources of one graph in one
launch give, source by source, the same distance and parent bits as the
single-source search -- on the renumbered SSSP copy and on the canonical
CSR, with repeated sources and roots in small components -- and pass the
SSSP validator; bad arguments are refused."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g16(cgt):
    return cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2, 3), 16, 16 << 16)


def _single(cgt, g, src):
    st = cgt.SsspState(g)
    out = []
    for r in src:
        cgt.oned_graph_sssp_run(g, st, int(r))
        cgt.sssp_status(st)
        out.append((st.dist.clone(), st.pred.clone()))
    return out


def test_multi_equals_single_source(cgt, g16):
    g = g16
    roots = cgt.generate_bfs_roots(g, 2, 3, 64)[:32]
    dist, pred, st = cgt.oned_graph_sssp_multi(g, roots)
    assert st.error_flags == 0 and st.rounds > 0
    for s, (d1, p1) in enumerate(_single(cgt, g, roots)):
        assert torch.equal(dist[s].view(torch.int32), d1.view(torch.int32)), s
        assert torch.equal(pred[s], p1), s
    vw = cgt._val_work(g)
    for s in (0, 7):
        assert cgt.sssp_validate(g, int(roots[s]), dist[s], pred[s], vw) == 0


def test_multi_on_canonical_csr_with_repeats(cgt, g16):
    g = g16
    deg = np.diff(g.rowstarts.cpu().numpy())
    small = [int(v) for v in np.nonzero(deg > 0)[0] if not g.in_main_component(int(v))][:2]
    main = [r for r in cgt.generate_bfs_roots(g, 5, 7, 8) if g.in_main_component(r)][:2]
    src = main + small + [main[0]]  # a source twice
    k, n = len(src), g.nglobalverts
    work = cgt.sssp_multi_workspace(g)
    dist = torch.empty((k, n), dtype=torch.float32, device="cuda")
    pred = torch.empty((k, n), dtype=torch.int64, device="cuda")
    h = (C.c_uint64 * k)(*src)
    st = cgt.SsspMultiStats()
    rc = cgt.lib.g5_sssp_multi_run(g.rowstarts.data_ptr(), g.col.data_ptr(), g.w.data_ptr(), n, None, None, h, k,
                                   dist.data_ptr(), pred.data_ptr(), work.data_ptr(), work.numel(), 0.0, 0,
                                   C.byref(st), None)
    assert rc == 0, cgt.lib.g5_last_error()
    for s, (d1, p1) in enumerate(_single(cgt, g, src)):
        assert torch.equal(dist[s].view(torch.int32), d1.view(torch.int32)), s
        assert torch.equal(pred[s], p1), s
    assert torch.equal(dist[0], dist[k - 1])
    # a small grid, and other bucket widths, give the same bits
    for kw in (dict(blocks=3), dict(delta=0.02), dict(delta=0.1), dict(delta=0.7)):
        d2, p2, _ = cgt.oned_graph_sssp_multi(g, src, work=work, **kw)
        assert torch.equal(d2.view(torch.int32), dist.view(torch.int32)) and torch.equal(p2, pred), kw


def test_multi_refuses_bad_arguments(cgt, g16):
    g = g16
    n = g.nglobalverts
    work = cgt.sssp_multi_workspace(g)
    lib = cgt.lib
    h = (C.c_uint64 * 33)(*range(33))
    args = (g.rowstarts.data_ptr(), g.col.data_ptr(), g.w.data_ptr(), n, None, None)
    run = lambda src, k, nbytes, delta=0.0: lib.g5_sssp_multi_run(*args, src, k, None, None, work.data_ptr(), nbytes,
                                                                  delta, 0, None, None)  # noqa: E731
    assert run(h, 0, work.numel()) == -1
    assert run(h, 33, work.numel()) == -1
    bad = (C.c_uint64 * 1)(n)
    assert run(bad, 1, work.numel()) == -1 and b"outside" in lib.g5_last_error()
    assert run(h, 1, work.numel(), -0.5) == -1 and b"width" in lib.g5_last_error()
    assert run(h, 1, 1024) == -2
