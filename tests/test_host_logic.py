"""Host-side logic of the batching layers, without a GPU: the autotuner's
cache, the serving trace generator and latency summary."""
from __future__ import annotations

import types

import numpy as np
import torch


def _fake_graph(n, rowstarts=None, nentries=30000):
    rs = torch.as_tensor(rowstarts if rowstarts is not None else np.arange(n + 1) * 2, dtype=torch.int64)
    return types.SimpleNamespace(device=torch.device("cpu"), nglobalverts=n, nlocaledges=nentries, rowstarts=rs)


def test_tuning_cache_round_trip(cgt, tmp_path):
    """Settings are keyed by device, kind and graph size and survive a reload."""
    from cgt_b200 import autotune as T
    fake, other = _fake_graph(1 << 10), _fake_graph(1 << 11)
    c = T.TuningCache(str(tmp_path / "t.json"))
    assert c.get("bfs", fake) is None
    c.put("bfs", fake, {"alpha": 10.0, "beta": 24.0, "blocks": 0})
    c2 = T.TuningCache(str(tmp_path / "t.json"))
    assert c2.get("bfs", fake)["alpha"] == 10.0 and c2.get("bfs", other) is None and c2.get("sssp", fake) is None
    assert T.bfs_params(c2.get("bfs", fake)).alpha == 10.0


def test_tile_descent_and_committed_cache(cgt):
    """Coordinate descent over the tile axes: each axis keeps its fastest
    value with the others at their best so far, and no setting is timed
    twice.  The committed cache holds a B200 SCALE 26 result whose knobs
    form valid parameters."""
    import json
    import os
    from cgt_b200 import autotune as T
    timed = []

    def time_of(k):  # a bowl: best at chunk 512, big_deg 256, lane_entries 8
        timed.append(tuple(sorted(k.items())))
        return abs(k["chunk"] - 512) + abs(k["big_deg"] - 256) / 4 + abs(k["lane_entries"] - 8) * 10

    base = dict(T.BFS_DEFAULT_TILES)
    ms, best, count = T._descend(time_of, base, T.BFS_TILES)
    assert (best["chunk"], best["big_deg"], best["lane_entries"]) == (512, 256, 8) and ms == 0
    assert count == len(timed) == len(set(timed))
    assert count == 1 + sum(len(set(v) - {base[k]}) for k, v in T.BFS_TILES.items())
    path = os.path.join(os.path.dirname(cgt.__file__), "tuned.json")
    data = json.load(open(path))
    kinds = {k.split("|")[1] for k in data}
    assert kinds == {"bfs", "sssp"} and all(k.startswith("NVIDIA B200|") for k in data)
    for key, t in data.items():
        if "|bfs|" in key:
            p = T.bfs_params(t)
            assert p.chunk % 32 == 0 and 0 < p.alpha and p.lane_entries % 4 == 0
        else:
            kw = T.sssp_kwargs(t)
            assert kw["delta"] == 0.1 and kw["chunk"] % 64 == 0


def test_poisson_trace_and_summary(cgt):
    from cgt_b200 import serve as S
    # graph 1 has isolated vertices 0 and 2: roots never land there
    g0 = _fake_graph(8)
    g1 = _fake_graph(4, rowstarts=[0, 0, 3, 3, 5])
    tr = S.poisson_trace([g0, g1], 2000, rate=1000.0, bfs_share=0.7, seed=5)
    assert len(tr) == 2000 and all(a.arrival < b.arrival for a, b in zip(tr, tr[1:]))
    assert 0.65 < sum(q.kind == "bfs" for q in tr) / len(tr) < 0.75
    assert {q.root for q in tr if q.graph == 1} <= {1, 3}
    assert abs(tr[-1].arrival - 2.0) < 0.3  # mean gap 1 ms
    assert tr == S.poisson_trace([g0, g1], 2000, rate=1000.0, bfs_share=0.7, seed=5)
    res = [S.Result(q.qid, q.kind, q.graph, q.root, q.arrival, q.arrival + 0.001 * (1 + q.qid % 10), 1)
           for q in tr]
    s = S.latency_summary(res)
    assert s["queries"] == 2000 and s["failed"] == 0 and abs(s["p50_ms"] - 5.5) < 1.0 and s["p99_ms"] >= 9.9
    # failed queries (ok=False) are counted apart, not in qps or the percentiles
    res[0] = S.Result(0, "bfs", 0, 1, res[0].arrival, res[0].arrival + 100.0, 1, None, False)
    f = S.latency_summary(res)
    assert f["queries"] == 1999 and f["failed"] == 1 and f["p99_ms"] < 20.0
    assert f["qps"] < s["qps"]  # the failed query still spans the makespan


def test_query_host_pointer_cache_and_sssp_params(cgt):
    """The query path looks up the host address of the main-component bitmap
    once per array (a new array gets a new address), and SSSP parameters carry
    the graph's tiny counts only when the graph has them."""
    n = 64
    rs = torch.arange(n + 1, dtype=torch.int64)
    g = cgt.OnedGraph(n, n, rs, torch.zeros(n, dtype=torch.int32), torch.zeros(n), torch.zeros(n, dtype=torch.int32),
                      0.1)
    assert cgt._main_bits_ptr(g) is None
    g.main_bits = np.full(2, 0xFFFFFFFF, np.uint32)
    a = cgt._main_bits_ptr(g)
    assert a == g.main_bits.ctypes.data and cgt._main_bits_ptr(g) == a
    g.main_bits = np.zeros(2, np.uint32)
    assert cgt._main_bits_ptr(g) == g.main_bits.ctypes.data
    p = cgt._sssp_params(g, 0, 0.1, 0, 0.0, 0, None)
    assert p.tiny_deg is None and p.small == 1 and p.blocks == 1  # root 0 outside the (empty) main component
    g.tiny_deg = torch.zeros(n, dtype=torch.int32)
    p = cgt._sssp_params(g, 0, 0.1, 0, 0.0, 0, False)
    assert p.tiny_deg == g.tiny_deg.data_ptr() and p.small == 0 and p.blocks == 0


def test_server_status_errors_counted_or_raised(cgt):
    """A launch whose status reports a device error raises by default; with
    raise_errors=False it is counted and the server goes on."""
    from cgt_b200 import serve as S

    def bad(resource, stream):
        raise cgt.G5Error("libg500b error -5: internal capacity exceeded")

    def good(resource, stream):
        return None

    srv = object.__new__(S.GraphServer)
    srv.stats = S.ServerStats()
    srv.raise_errors = True
    assert srv._checked(good, None, None)
    try:
        srv._checked(bad, None, None)
        raise AssertionError("expected G5Error")
    except cgt.G5Error:
        pass
    srv.raise_errors = False
    assert not srv._checked(bad, None, None) and srv.stats.device_errors == 1 and len(srv.stats.errors) == 1

    # The library's device errors are G5Error subclasses (and their builtin kinds).
    def timeout(resource, stream):
        raise cgt._ERRORS[-4]("libg500b error -4: a bounded grid barrier wait expired")

    def device(resource, stream):
        raise cgt._ERRORS[-5]("libg500b error -5: internal capacity exceeded")

    assert issubclass(cgt._ERRORS[-4], TimeoutError) and issubclass(cgt._ERRORS[-1], ValueError)
    assert not srv._checked(timeout, None, None) and not srv._checked(device, None, None)
    assert srv.stats.device_errors == 3
