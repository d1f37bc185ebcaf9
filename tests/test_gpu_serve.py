"""The query server (serve.py): continuous batching over resident graphs
returns, for every query, exactly what the query computes alone."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graphs(cgt):
    return [cgt.oned_graph_from_kronecker(cgt.make_mrg_seed(2 + i, 3), s, 16 << s, with_main=False)
            for i, s in enumerate((10, 12, 14, 12))]


def test_batched_results_equal_alone(cgt, graphs):
    from cgt_b200 import serve
    trace = serve.poisson_trace(graphs, 300, rate=20000.0, bfs_share=0.7, seed=3)
    srv = serve.GraphServer(graphs, slots=4, hbm_reserve=1 << 30, keep_results=True)
    srv.prewarm()
    assert all(srv.sssp_free[gi] and srv.bfs_free[gi] for gi in range(len(graphs)))
    res = srv.run_trace(trace, deadline=120.0)
    assert sorted(r.qid for r in res) == list(range(300))
    assert srv.stats.bfs_batches < sum(1 for q in trace if q.kind == "bfs")  # queries were batched
    assert srv.stats.sssp_batches > 0 and srv.stats.sssp_batched_queries > srv.stats.sssp_batches  # SSSP too
    assert max(r.batch for r in res) > 1
    alone = {r.qid: r for r in serve.serve_plain(graphs, trace, keep_results=True)}
    for r in res:
        a = alone[r.qid]
        if r.kind == "bfs":
            assert torch.equal(r.value, a.value), r.qid
        else:
            assert torch.equal(r.value.view(torch.int32), a.value.view(torch.int32)), r.qid
    s = serve.latency_summary(res)
    assert s["queries"] == 300 and s["p99_ms"] >= s["p50_ms"] > 0


def test_few_bfs_queries_run_single(cgt, graphs):
    """Fewer than bfs_batch_min waiting BFS queries of a graph take the plain
    single-root search, with the same depth arrays."""
    from cgt_b200 import serve
    trace = [serve.Query(i, "bfs", i % len(graphs), 1 + 7 * i, 0.002 * i) for i in range(6)]
    srv = serve.GraphServer(graphs, slots=4, hbm_reserve=1 << 30, keep_results=True)
    res = srv.run_trace(trace, deadline=60.0)
    assert srv.stats.bfs_single > 0
    alone = {r.qid: r for r in serve.serve_plain(graphs, trace, keep_results=True)}
    for r in res:
        assert torch.equal(r.value, alone[r.qid].value), r.qid


def test_small_graph_searches_overlap(cgt, graphs):
    """SSSP queries on small graphs use small grids and run side by side."""
    from cgt_b200 import serve
    trace = [serve.Query(i, "sssp", 0, int(r), 0.0) for i, r in
             enumerate(np.nonzero(np.diff(graphs[0].rowstarts.cpu().numpy()) > 0)[0][:40])]
    srv = serve.GraphServer(graphs, slots=4, hbm_reserve=1 << 30)
    srv.run_trace(trace, deadline=60.0)
    assert srv.stats.max_inflight > 1


def test_admission_waits_for_memory(cgt, graphs):
    """With no device memory to spare, nothing is admitted: the work waits
    (here until the deadline) instead of over-allocating."""
    from cgt_b200 import serve
    _, total = torch.cuda.mem_get_info()
    srv = serve.GraphServer(graphs, hbm_reserve=total)
    with pytest.raises(TimeoutError):
        srv.run_trace([serve.Query(0, "bfs", 1, 5, 0.0)], deadline=0.5)
    assert srv.stats.refused_for_memory > 0 and srv.stats.launches == 0
    with pytest.raises(ValueError):
        srv.submit(serve.Query(1, "bfs", 9, 0, 0.0))
