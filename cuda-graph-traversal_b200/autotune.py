"""Autotuner for the run-time knobs of the persistent searches: the BFS
direction thresholds (alpha, beta), the batched BFS's switch threshold and
frontier test, the SSSP bucket width delta, each kernel's grid size
(blocks per launch), and the work tiles: the row length above which a list
entry is cut into chunks spread over the grid, the chunk size, and the BFS
bottom-up lane scan length.  No counterpart in the reference, which fixes its launch shape and
delta (src/traversal.cu:479-503, 638-711).

Every candidate is timed on the device (CUDA events, the search alone, its
reset outside the timer) over a few roots of the caller's graph; the fastest
total wins.  None of the knobs changes a result: BFS depths, batched depths
and SSSP distances are the same for every setting (the GPU tests check
that), so the tuner only trades speed.  Results can be kept in a JSON file
keyed by device, search kind and graph size.
"""
from __future__ import annotations

import itertools
import json
import os

import torch

from . import (BfsParams, BfsState, MsBfsParams, MsBfsState, OnedGraph, SsspState, msbfs_run, oned_graph_bfs_reset,
               oned_graph_bfs_traverse, oned_graph_bfs_traverse_multi, oned_graph_sssp_reset,
               oned_graph_sssp_traverse, oned_graph_sssp_traverse_multi, search_grid)


def _timed(enqueue, reset=None) -> float:
    """Device milliseconds of enqueue() (reset() runs first, untimed)."""
    if reset is not None:
        reset()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    enqueue()
    b.record()
    b.synchronize()
    return a.elapsed_time(b)


def _grids(kind: str, n: int) -> list[int]:
    """Default grid plus the full device and fractions of it."""
    b, m = search_grid(kind, n)
    return sorted({0, m, max(1, m // 2), max(1, m // 4), b})


def _searches(roots):
    """A tensor of roots is one multi-root search; a list is one search each."""
    return [roots] if isinstance(roots, torch.Tensor) else [int(r) for r in roots]


def _descend(time_of, base: dict, axes: dict) -> tuple[float, dict, int]:
    """Coordinate descent over the tile axes: each axis in turn takes the
    value that times fastest with the others held at their best so far.
    Returns (ms, settings, candidates timed)."""
    best = dict(base)
    best_ms = time_of(best)
    count = 1
    for name, values in axes.items():
        tried = {best[name]}  # timed already, as part of best
        for v in values:
            if v in tried:
                continue
            tried.add(v)
            trial = dict(best, **{name: v})
            ms = time_of(trial)
            count += 1
            if ms < best_ms:
                best_ms, best = ms, trial
    return best_ms, best, count


BFS_TILES = {"chunk": (128, 256, 512, 1024), "big_deg": (256, 1024, 4096), "lane_entries": (4, 8, 16, 32)}
SSSP_TILES = {"chunk": (128, 256, 512, 1024), "big_deg": (64, 128, 256, 512)}
# The library's defaults (what 0 in g5_bfs_params / g5_sssp_params selects).
BFS_DEFAULT_TILES = {"big_deg": 1024, "chunk": 256, "lane_entries": 8}
SSSP_DEFAULT_TILES = {"big_deg": 256, "chunk": 256}


def tune_bfs(g: OnedGraph, roots, alphas=(6.0, 10.0, 14.0, 20.0, 28.0), betas=(12.0, 24.0, 48.0), grids=None,
             reps: int = 1, tiles: dict | None = BFS_TILES) -> dict:
    """Best (alpha, beta, blocks) for BFS over `roots`: a list of roots (one
    search each) or a device tensor (one multi-root search, as on packed
    graphs); then, with those fixed, the work tiles of g5_bfs_params
    (big_deg, chunk, lane_entries) by coordinate descent over `tiles`
    (None: the library's defaults)."""
    bfs = BfsState(g)
    grids = _grids("bfs", g.nglobalverts) if grids is None else list(grids)

    def time_of(k: dict) -> float:
        p = BfsParams(k["alpha"], k["beta"], 0, k["blocks"], k.get("big_deg", 0), k.get("chunk", 0),
                      k.get("lane_entries", 0))
        ms = 0.0
        for _ in range(reps):
            for r in _searches(roots):
                if isinstance(r, torch.Tensor):
                    run = lambda: oned_graph_bfs_traverse_multi(g, bfs, r, p, with_depth=False)  # noqa: E731
                else:
                    run = lambda: oned_graph_bfs_traverse(g, bfs, r, p, with_depth=False)  # noqa: E731
                ms += _timed(run, lambda: oned_graph_bfs_reset(bfs, False, g))
        return ms / reps

    table = [(time_of({"alpha": a, "beta": b, "blocks": k}), a, b, k)
             for a, b, k in itertools.product(alphas, betas, grids)]
    best = min(table)
    out = {"alpha": best[1], "beta": best[2], "blocks": best[3], "big_deg": 0, "chunk": 0, "lane_entries": 0}
    ms, count = best[0], len(table)
    if tiles:
        out.update(**BFS_DEFAULT_TILES)  # the library's defaults, spelled out
        ms, out, more = _descend(time_of, out, tiles)
        count += more
    return {"kind": "bfs", **out, "ms": round(ms, 4), "candidates": count}


def tune_sssp(g: OnedGraph, roots, deltas=(0.08, 0.1, 0.2, 0.4), grids=None, pulls=(0.0, -1.0), subs=(0, -1),
              reps: int = 1, tiles: dict | None = SSSP_TILES) -> dict:
    """Best (delta, blocks, pull, sub_min) for SSSP over `roots` (a list: one
    search each; a device tensor: one multi-source search).  pull / sub_min
    are g5_sssp_params' heavy-phase pull threshold and sub-bucket threshold
    (0 = the library's default, -1 = off).  Then the list tiles (big_deg,
    chunk) by coordinate descent over `tiles`."""
    st = SsspState(g)
    grids = _grids("sssp", g.nglobalverts) if grids is None else list(grids)

    def time_of(k: dict) -> float:
        kw = dict(big_deg=k.get("big_deg", 0), chunk=k.get("chunk", 0))
        ms = 0.0
        for _ in range(reps):
            for r in _searches(roots):
                if isinstance(r, torch.Tensor):
                    run = lambda: oned_graph_sssp_traverse_multi(g, st, r, k["delta"], k["blocks"], k["pull"],  # noqa: E731
                                                                 k["sub_min"], **kw)
                else:
                    run = lambda: oned_graph_sssp_traverse(g, st, r, k["delta"], k["blocks"], k["pull"],  # noqa: E731
                                                           k["sub_min"], **kw)
                ms += _timed(run, lambda: oned_graph_sssp_reset(st))
        return ms / reps

    table = [(time_of({"delta": d, "blocks": b, "pull": p, "sub_min": s}), d, b, p, s)
             for d, b, p, s in itertools.product(deltas, grids, pulls, subs)]
    best = min(table)
    out = {"delta": best[1], "blocks": best[2], "pull": best[3], "sub_min": best[4], "big_deg": 0, "chunk": 0}
    ms, count = best[0], len(table)
    if tiles:
        out.update(**SSSP_DEFAULT_TILES)
        ms, out, more = _descend(time_of, out, tiles)
        count += more
    return {"kind": "sssp", **out, "ms": round(ms, 4), "candidates": count}


def tune_msbfs(g: OnedGraph, roots, alphas=(8.0, 16.0, 32.0, 64.0), checks=(0, 1, 2), grids=None,
               ms: MsBfsState | None = None, reps: int = 1) -> dict:
    """Best (alpha, check_frontier, blocks) for one batched search of `roots`."""
    ms = MsBfsState(g) if ms is None else ms
    grids = [0] if grids is None else list(grids)
    table = []
    for alpha, check, blocks in itertools.product(alphas, checks, grids):
        p = MsBfsParams(alpha, 0, check, blocks)
        t = min(_timed(lambda: msbfs_run(g, ms, roots, p, sync=False)) for _ in range(reps))
        table.append((t, alpha, check, blocks))
    best = min(table)
    return {"kind": "msbfs", "alpha": best[1], "check_frontier": best[2], "blocks": best[3], "ms": round(best[0], 4),
            "candidates": len(table)}


def bfs_params(t: dict) -> BfsParams:
    return BfsParams(t["alpha"], t["beta"], 0, t["blocks"], t.get("big_deg", 0), t.get("chunk", 0),
                     t.get("lane_entries", 0))


def sssp_kwargs(t: dict) -> dict:
    """Keyword arguments of oned_graph_sssp_run / _traverse for a tune_sssp result."""
    return {k: t.get(k, 0) for k in ("delta", "blocks", "pull", "sub_min", "big_deg", "chunk")}


def msbfs_params(t: dict) -> MsBfsParams:
    return MsBfsParams(t["alpha"], 0, t["check_frontier"], t["blocks"])


class TuningCache:
    """Tuned settings in a JSON file, keyed by device name, search kind and
    graph size (vertices, CSR entries)."""

    def __init__(self, path: str):
        self.path = path
        self.data = {}
        if os.path.exists(path):
            with open(path) as f:
                self.data = json.load(f)

    @staticmethod
    def key(kind: str, g: OnedGraph) -> str:
        dev = torch.cuda.get_device_name(g.device) if g.device.type == "cuda" else str(g.device)
        return f"{dev}|{kind}|n={g.nglobalverts}|e={g.nlocaledges}"

    def get(self, kind: str, g: OnedGraph) -> dict | None:
        return self.data.get(self.key(kind, g))

    def put(self, kind: str, g: OnedGraph, result: dict) -> None:
        self.data[self.key(kind, g)] = result
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    def tuned(self, kind: str, g: OnedGraph, roots, **kw) -> dict:
        """Cached result, or tune now (tune_bfs / tune_sssp / tune_msbfs) and keep it."""
        hit = self.get(kind, g)
        if hit is None:
            hit = {"bfs": tune_bfs, "sssp": tune_sssp, "msbfs": tune_msbfs}[kind](g, roots, **kw)
            self.put(kind, g, hit)
        return hit
