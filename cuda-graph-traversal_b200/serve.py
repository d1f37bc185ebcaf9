"""Query serving over graphs resident on one GPU: continuous batching of BFS
and SSSP queries.  No counterpart in the reference, whose runner issues one
search per call (examples/graph500_runner.cu:303-409).

A query asks for every vertex's BFS depth or SSSP distance from a root of
one resident graph.  The server keeps per graph a pending BFS queue and a
pending SSSP queue and a pool of CUDA streams ("slots").  Whenever a slot is
free it launches the oldest waiting work:

* all pending BFS queries of a graph (up to 256) become one batched search
  (g5_msbfs_run + depth export) on that graph's batched-BFS workspace --
  when at least `bfs_batch_min` (8) are waiting; fewer are answered one at a
  time by the plain search on a pooled BFS workspace, which costs less than
  a batched search below about 8 roots (SCALE 16-24: a batch of one root
  takes 4-6x a plain search, a batch of 16 about 1.1x two plain searches);
* pending SSSP queries of a graph of at most `sssp_batch_max_vertices`
  (2^20) vertices, when at least `sssp_batch_min` (2) wait, become one
  batched search of up to 32 sources (g5_sssp_multi_run) on that graph's
  batched-SSSP workspace, which answers 32 sources 1.5-13x faster than 32
  single searches on graphs of 2^20 down to 2^14 vertices; otherwise (and on
  larger graphs, where the single search is the faster one) an SSSP query
  runs on its own on a pooled SSSP workspace of that graph.

Every search is a persistent cooperative kernel whose grid is sized to its
graph (g5_*_grid); launches run concurrently only while the sum of their
grids fits on the device at once, so no two grids can wait on each other
for SMs, and small graphs' searches share the GPU.  A launch gets at most
1/k of the device, k = the launches running plus the queue heads waiting
(at most `slots`): a search on a quarter of the SMs takes well under four
times as long (its phases are latency bound), so under load several
searches side by side answer more queries per second, while a lone query
still gets the whole device.

Queries that arrive while others run join the next batch of their graph, so
batches form continuously and work on different graphs and different
queries overlaps on the device.  Workspaces are created on first use and
only while free device memory stays above `hbm_reserve` (admission by free
HBM); otherwise the work waits for a workspace to come free.  Completion is
seen by polling each launch's CUDA event.  A query's result (an int32 depth
array, -1 unreached, or a float32 distance array, -1.0 unreached) is
identical whether it ran alone or in a batch.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import (MSBFS_MAX_ROOTS, BfsParams, BfsState, G5Error, MsBfsParams, MsBfsState, OnedGraph,
               SsspMultiState, SsspState, bfs_stats, bfs_workspace_bytes, msbfs_depths_u8, msbfs_run, msbfs_stats,
               oned_graph_bfs_reset, oned_graph_bfs_run, oned_graph_bfs_traverse, oned_graph_sssp_multi,
               oned_graph_sssp_reset, oned_graph_sssp_traverse, search_grid, sssp_multi_status, sssp_status,
               sssp_workspace_bytes)

SSSP_BATCH_MAX = 32  # sources of one batched SSSP launch


@dataclass
class Query:
    qid: int
    kind: str      # "bfs" or "sssp"
    graph: int     # index into the server's graphs
    root: int
    arrival: float = 0.0  # seconds, on the trace's clock


@dataclass
class Result:
    qid: int
    kind: str
    graph: int
    root: int
    arrival: float
    done: float           # seconds, same clock as arrival
    batch: int            # queries in the launch that answered it
    value: torch.Tensor | None = None  # depth (int32) or distance (float32), when kept
    ok: bool = True       # False: the launch reported a device error (its result is not valid)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class _Launch:
    event: torch.cuda.Event
    queries: list
    kind: str
    graph: int
    slot: int
    resource: object
    blocks: int
    out: torch.Tensor | None = None


@dataclass
class ServerStats:
    launches: int = 0
    bfs_batches: int = 0
    bfs_batched_queries: int = 0
    bfs_single: int = 0
    sssp_launches: int = 0
    sssp_batches: int = 0
    sssp_batched_queries: int = 0
    max_inflight: int = 0
    workspaces: dict = field(default_factory=dict)
    refused_for_memory: int = 0
    device_errors: int = 0                           # launches whose status reported an error
    errors: list = field(default_factory=list)       # the first few messages


class GraphServer:
    def __init__(self, graphs: list[OnedGraph], slots: int = 4, hbm_reserve: int = 8 << 30,
                 max_batch: int = MSBFS_MAX_ROOTS, keep_results: bool = False, max_sssp_per_graph: int = 4,
                 bfs_batch_min: int = 8, raise_errors: bool = True, sssp_batch_min: int = 2,
                 sssp_batch_max_vertices: int = 1 << 20):
        if not graphs:
            raise ValueError("GraphServer needs at least one graph")
        self.graphs = graphs
        self.dev = graphs[0].device
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(slots)]
        self.free_slots = list(range(slots))
        self.hbm_reserve = int(hbm_reserve)
        self.max_batch = int(max_batch)
        self.keep = keep_results
        self.raise_errors = raise_errors
        self.max_sssp = int(max_sssp_per_graph)
        self.bfs_batch_min = max(1, int(bfs_batch_min))
        self.bfs_free: list[list[BfsState]] = [[] for _ in graphs]
        self.bfs_count = [0] * len(graphs)
        self.pending = {k: [collections.deque() for _ in graphs] for k in ("bfs", "sssp")}
        self.ms: list[MsBfsState | None] = [None] * len(graphs)
        self.ms_busy = [False] * len(graphs)
        self.sssp_free: list[list[SsspState]] = [[] for _ in graphs]
        self.sssp_count = [0] * len(graphs)
        self.sssp_batch_min = max(2, int(sssp_batch_min))
        self.sssp_batch_max_vertices = int(sssp_batch_max_vertices)
        self.mss: list[SsspMultiState | None] = [None] * len(graphs)
        self.mss_busy = [False] * len(graphs)
        self.inflight: list[_Launch] = []
        kinds = ("bfs", "msbfs", "sssp", "sssp_multi")
        self.grid = {k: [search_grid(k, g.nglobalverts)[0] for g in graphs] for k in kinds}
        self.max_blocks = min(search_grid(k, 1)[1] for k in kinds)
        self.blocks_in_use = 0
        self.stats = ServerStats()
        self.clock0 = time.perf_counter()

    # ------------------------------------------------------------ admission
    def _fits(self, nbytes: int) -> bool:
        free, _ = torch.cuda.mem_get_info(self.dev)
        ok = free - nbytes >= self.hbm_reserve
        if not ok:
            self.stats.refused_for_memory += 1
        return ok

    def _ms_state(self, gi: int) -> MsBfsState | None:
        if self.ms[gi] is None:
            g = self.graphs[gi]
            need = 330 * g.nglobalverts + 12 * g.nlocaledges  # rows, planes, renumbered copy
            if not self._fits(need):
                return None
            self.ms[gi] = MsBfsState(g)
            self.stats.workspaces[f"msbfs{gi}"] = self.ms[gi].work.numel()
        return self.ms[gi]

    def _mss_state(self, gi: int) -> SsspMultiState | None:
        """The graph's batched-SSSP workspace (graphs up to
        sssp_batch_max_vertices only)."""
        g = self.graphs[gi]
        if g.nglobalverts > self.sssp_batch_max_vertices:
            return None
        if self.mss[gi] is None:
            if not self._fits(404 * g.nglobalverts):  # workspace + 32 distance rows
                return None
            self.mss[gi] = SsspMultiState(g, SSSP_BATCH_MAX)
            self.stats.workspaces[f"sssp_multi{gi}"] = self.mss[gi].work.numel()
        return self.mss[gi]

    def _bfs_state(self, gi: int) -> BfsState | None:
        if self.bfs_free[gi]:
            return self.bfs_free[gi].pop()
        return self._new_bfs_state(gi)

    def _new_bfs_state(self, gi: int) -> BfsState | None:
        if self.bfs_count[gi] >= self.max_sssp:
            return None
        g = self.graphs[gi]
        if not self._fits(bfs_workspace_bytes(g.nglobalverts) + 12 * g.nglobalverts):  # + pred, depth
            return None
        self.bfs_count[gi] += 1
        self.stats.workspaces[f"bfs{gi}_{self.bfs_count[gi]}"] = 1
        return BfsState(g)

    def _sssp_state(self, gi: int) -> SsspState | None:
        if self.sssp_free[gi]:
            return self.sssp_free[gi].pop()
        return self._new_sssp_state(gi)

    def _new_sssp_state(self, gi: int) -> SsspState | None:
        if self.sssp_count[gi] >= self.max_sssp:
            return None
        g = self.graphs[gi]
        if not self._fits(sssp_workspace_bytes(g.nglobalverts) + 12 * g.nglobalverts):  # + dist, pred
            return None
        self.sssp_count[gi] += 1
        self.stats.workspaces[f"sssp{gi}_{self.sssp_count[gi]}"] = 1
        return SsspState(g)

    def prewarm(self) -> None:
        """Creates the workspaces a trace can use -- per graph the batched-BFS
        workspace, then plain BFS and SSSP workspaces up to the per-graph cap,
        round-robin over the graphs -- while admission by free HBM allows, so
        that no query waits on a first-use allocation."""
        for gi in range(len(self.graphs)):
            self._ms_state(gi)
            self._mss_state(gi)
        for _ in range(self.max_sssp):
            grew = False
            for gi in range(len(self.graphs)):
                for make, free in ((self._new_bfs_state, self.bfs_free), (self._new_sssp_state, self.sssp_free)):
                    st = make(gi)
                    if st is not None:
                        free[gi].append(st)
                        grew = True
            if not grew:
                break

    # ------------------------------------------------------------- queueing
    def now(self) -> float:
        return time.perf_counter() - self.clock0

    def submit(self, q: Query) -> None:
        if q.kind not in ("bfs", "sssp"):
            raise ValueError(f"unknown query kind {q.kind!r}")
        if not 0 <= q.graph < len(self.graphs):
            raise ValueError(f"query {q.qid}: no graph {q.graph}")
        if not 0 <= q.root < self.graphs[q.graph].nglobalverts:
            raise ValueError(f"query {q.qid}: root {q.root} out of range")
        self.pending[q.kind][q.graph].append(q)

    def idle(self) -> bool:
        return not self.inflight and not any(any(d) for k in self.pending.values() for d in k)

    def _candidates(self):
        """(arrival, kind, graph) of every launchable queue head, oldest first."""
        c = []
        for kind, queues in self.pending.items():
            for gi, d in enumerate(queues):
                if d and not (kind == "bfs" and self.ms_busy[gi]):
                    c.append((d[0].arrival, kind, gi))
        c.sort()
        return c

    # --------------------------------------------------------------- launch
    def _launch_one(self) -> bool:
        """Launches the oldest work whose grid fits beside what runs; work
        without a workspace (memory) is passed over.  False when nothing
        could start."""
        if not self.free_slots:
            return False
        cands = self._candidates()
        k = min(len(self.streams), len(self.inflight) + len(cands))
        share = max(1, self.max_blocks // max(1, k))
        for _, kind, gi in cands:
            single = kind == "bfs" and len(self.pending["bfs"][gi]) < self.bfs_batch_min
            sbatch = (kind == "sssp" and len(self.pending["sssp"][gi]) >= self.sssp_batch_min and not self.mss_busy[gi]
                      and self._mss_state(gi) is not None)
            gk = ("bfs" if single else "msbfs") if kind == "bfs" else ("sssp_multi" if sbatch else "sssp")
            blocks = min(self.grid[gk][gi], share)
            if self.blocks_in_use + blocks > self.max_blocks:
                # Oldest first: younger work may not take the SMs this
                # launch is waiting for (a full-device search would starve).
                return False
            g = self.graphs[gi]
            if single:
                st = self._bfs_state(gi)
                if st is None:
                    continue
                slot = self.free_slots.pop()
                q = self.pending["bfs"][gi].popleft()
                s = self.streams[slot]
                with torch.cuda.stream(s):
                    oned_graph_bfs_reset(st, True, g, stream=s)
                    oned_graph_bfs_traverse(g, st, q.root, BfsParams(14.0, 24.0, 0, blocks), True, stream=s)
                    ev = torch.cuda.Event()
                    ev.record(s)
                self.inflight.append(_Launch(ev, [q], "bfs1", gi, slot, st, blocks))
                self.stats.bfs_single += 1
            elif kind == "bfs":
                ms = self._ms_state(gi)
                if ms is None:
                    continue
                slot = self.free_slots.pop()
                d = self.pending["bfs"][gi]
                qs = [d.popleft() for _ in range(min(len(d), self.max_batch))]
                s = self.streams[slot]
                with torch.cuda.stream(s):
                    msbfs_run(g, ms, [q.root for q in qs], MsBfsParams(0.0, 0, 0, blocks), sync=False, stream=s)
                    out = msbfs_depths_u8(ms, stream=s)
                    ev = torch.cuda.Event()
                    ev.record(s)
                self.ms_busy[gi] = True
                self.inflight.append(_Launch(ev, qs, "bfs", gi, slot, ms, blocks, out))
                self.stats.bfs_batches += 1
                self.stats.bfs_batched_queries += len(qs)
            elif sbatch:
                ms = self.mss[gi]
                slot = self.free_slots.pop()
                d = self.pending["sssp"][gi]
                qs = [d.popleft() for _ in range(min(len(d), SSSP_BATCH_MAX))]
                s = self.streams[slot]
                with torch.cuda.stream(s):
                    oned_graph_sssp_multi(g, [q.root for q in qs], work=ms.work, with_pred=False, blocks=blocks,
                                          stream=s, dist=ms.dist[:len(qs)], sync=False)
                    ev = torch.cuda.Event()
                    ev.record(s)
                self.mss_busy[gi] = True
                self.inflight.append(_Launch(ev, qs, "sssp_b", gi, slot, ms, blocks))
                self.stats.sssp_batches += 1
                self.stats.sssp_batched_queries += len(qs)
            else:
                st = self._sssp_state(gi)
                if st is None:
                    continue
                slot = self.free_slots.pop()
                q = self.pending["sssp"][gi].popleft()
                s = self.streams[slot]
                with torch.cuda.stream(s):
                    oned_graph_sssp_reset(st, stream=s)
                    oned_graph_sssp_traverse(g, st, q.root, blocks=blocks, stream=s)
                    ev = torch.cuda.Event()
                    ev.record(s)
                self.inflight.append(_Launch(ev, [q], "sssp", gi, slot, st, blocks))
                self.stats.sssp_launches += 1
            self.blocks_in_use += blocks
            self.stats.launches += 1
            self.stats.max_inflight = max(self.stats.max_inflight, len(self.inflight))
            return True
        return False

    def _checked(self, status, resource, stream, launch=None) -> bool:
        """Reads a finished launch's status.  A device error raises, or with
        raise_errors=False is counted (the launch's queries are answered with
        ok=False) and the server goes on: the next reset clears the state.
        The message names the launch and what else was running."""
        try:
            status(resource, stream)
            return True
        except G5Error as ex:
            msg = str(ex)
            if launch is not None:
                others = [(x.kind, x.graph, x.blocks) for x in self.inflight if x is not launch]
                msg += f" [{launch.kind} graph {launch.graph} blocks {launch.blocks}; also running {others}]"
            if self.raise_errors:
                raise type(ex)(msg) from ex
            self.stats.device_errors += 1
            if len(self.stats.errors) < 8:
                self.stats.errors.append(msg)
            return False

    def _complete(self, L: _Launch, t: float) -> list[Result]:
        out = []
        if L.kind == "bfs1":
            ok = self._checked(bfs_stats, L.resource, self.streams[L.slot], L)
            q = L.queries[0]
            v = L.resource.depth.clone() if self.keep and ok else None
            out.append(Result(q.qid, "bfs", q.graph, q.root, q.arrival, t, 1, v, ok))
            self.bfs_free[L.graph].append(L.resource)
        elif L.kind == "bfs":
            ok = self._checked(msbfs_stats, L.resource, self.streams[L.slot], L)
            for i, q in enumerate(L.queries):
                v = None
                if self.keep and ok:
                    v = L.out[i].to(torch.int32)
                    v[v == 255] = -1
                out.append(Result(q.qid, q.kind, q.graph, q.root, q.arrival, t, len(L.queries), v, ok))
            self.ms_busy[L.graph] = False
        elif L.kind == "sssp_b":
            ok = self._checked(sssp_multi_status, L.resource, self.streams[L.slot], L)
            for i, q in enumerate(L.queries):
                v = L.resource.dist[i].clone() if self.keep and ok else None
                out.append(Result(q.qid, q.kind, q.graph, q.root, q.arrival, t, len(L.queries), v, ok))
            self.mss_busy[L.graph] = False
        else:
            ok = self._checked(sssp_status, L.resource, self.streams[L.slot], L)
            q = L.queries[0]
            v = L.resource.dist.clone() if self.keep and ok else None
            out.append(Result(q.qid, q.kind, q.graph, q.root, q.arrival, t, 1, v, ok))
            self.sssp_free[L.graph].append(L.resource)
        self.free_slots.append(L.slot)
        self.blocks_in_use -= L.blocks
        return out

    def poll(self) -> list[Result]:
        """Launches what it can, then collects finished launches."""
        while self._launch_one():
            pass
        done, still = [], []
        for L in self.inflight:
            if L.event.query():
                done.append(L)
            else:
                still.append(L)
        self.inflight = still
        t = self.now()
        res = []
        for L in done:
            res.extend(self._complete(L, t))
        if done:
            while self._launch_one():
                pass
        return res

    def run_trace(self, queries: list[Query], deadline: float | None = None) -> list[Result]:
        """Replays `queries` (sorted by arrival, seconds from now) in real
        time: each is submitted once its arrival time has passed.  Raises
        TimeoutError when work is still waiting `deadline` seconds after the
        start (for instance when no workspace can ever be admitted)."""
        queries = sorted(queries, key=lambda q: q.arrival)
        self.clock0 = time.perf_counter()
        results: list[Result] = []
        i = 0
        while i < len(queries) or not self.idle():
            t = self.now()
            if deadline is not None and t > deadline:
                raise TimeoutError(f"{len(queries) - len(results)} queries unanswered after {deadline} s "
                                   f"({self.stats.refused_for_memory} workspace requests refused for memory)")
            while i < len(queries) and queries[i].arrival <= t:
                self.submit(queries[i])
                i += 1
            results.extend(self.poll())
            if not self.inflight and i < len(queries) and not any(
                    any(d) for k in self.pending.values() for d in k):
                # nothing to do until the next arrival
                wait = queries[i].arrival - self.now()
                if wait > 0:
                    time.sleep(min(wait, 0.001))
        return results


def serve_plain(graphs: list[OnedGraph], queries: list[Query], keep_results: bool = False) -> list[Result]:
    """The same trace answered one query at a time with the plain calls
    (g5_bfs_run with depth, g5_sssp_run), in arrival order: a query starts
    when it has arrived and the previous one finished."""
    queries = sorted(queries, key=lambda q: q.arrival)
    bfs = [None] * len(graphs)
    sssp = [None] * len(graphs)
    t0 = time.perf_counter()
    out = []
    for q in queries:
        now = time.perf_counter() - t0
        if q.arrival > now:
            time.sleep(q.arrival - now)
        g = graphs[q.graph]
        if q.kind == "bfs":
            if bfs[q.graph] is None:
                bfs[q.graph] = BfsState(g)
            oned_graph_bfs_run(g, bfs[q.graph], q.root)
            torch.cuda.synchronize()
            v = bfs[q.graph].depth.clone() if keep_results else None
        else:
            if sssp[q.graph] is None:
                sssp[q.graph] = SsspState(g)
            oned_graph_sssp_reset(sssp[q.graph])
            oned_graph_sssp_traverse(g, sssp[q.graph], q.root)
            torch.cuda.synchronize()
            v = sssp[q.graph].dist.clone() if keep_results else None
        out.append(Result(q.qid, q.kind, q.graph, q.root, q.arrival, time.perf_counter() - t0, 1, v))
    return out


def poisson_trace(graphs: list[OnedGraph], nqueries: int, rate: float, bfs_share: float = 0.7,
                  seed: int = 1) -> list[Query]:
    """nqueries queries with exponential inter-arrival times (mean 1/rate
    seconds), kind BFS with probability bfs_share, graph uniform, root
    uniform over the graph's vertices of non-zero degree."""
    rng = np.random.default_rng(seed)
    nz = []
    for g in graphs:
        deg = (g.rowstarts[1:] - g.rowstarts[:-1]).cpu().numpy()
        nz.append(np.nonzero(deg > 0)[0])
    t = np.cumsum(rng.exponential(1.0 / rate, nqueries))
    kinds = np.where(rng.random(nqueries) < bfs_share, "bfs", "sssp")
    gsel = rng.integers(0, len(graphs), nqueries)
    qs = []
    for i in range(nqueries):
        cand = nz[gsel[i]]
        root = int(cand[rng.integers(0, len(cand))]) if len(cand) else 0
        qs.append(Query(i, str(kinds[i]), int(gsel[i]), root, float(t[i])))
    return qs


def latency_summary(results: list[Result]) -> dict:
    """Throughput and latency over the answered queries (ok); queries whose
    launch reported a device error are counted apart under "failed" and do
    not count towards qps or the percentiles.  The makespan runs from the
    first arrival to the last completion of any query."""
    good = [r for r in results if r.ok]
    span = max(r.done for r in results) - min(r.arrival for r in results)
    out = {"queries": len(good), "failed": len(results) - len(good), "qps": round(len(good) / span, 1),
           "makespan_s": round(span, 3)}
    if good:
        lat = np.array([r.latency for r in good])
        out.update({"p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 3),
                    "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 3),
                    "mean_ms": round(float(lat.mean()) * 1e3, 3)})
    else:
        out.update({"p50_ms": None, "p99_ms": None, "mean_ms": None})
    return out
