"""Autotuner for the run-time knobs of the persistent searches: the BFS
direction thresholds (alpha, beta), the batched BFS's switch threshold and
frontier test, the SSSP bucket width delta, and each kernel's grid size
(blocks per launch -- the tile of work the persistent grid cuts a level
into).  No counterpart in the reference, which fixes its launch shape and
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


def tune_bfs(g: OnedGraph, roots, alphas=(6.0, 10.0, 14.0, 20.0, 28.0), betas=(12.0, 24.0, 48.0), grids=None,
             reps: int = 1) -> dict:
    """Best (alpha, beta, blocks) for BFS over `roots`: a list of roots (one
    search each) or a device tensor (one multi-root search, as on packed
    graphs)."""
    bfs = BfsState(g)
    grids = _grids("bfs", g.nglobalverts) if grids is None else list(grids)
    table = []
    for alpha, beta, blocks in itertools.product(alphas, betas, grids):
        p = BfsParams(alpha, beta, 0, blocks)
        ms = 0.0
        for _ in range(reps):
            for r in _searches(roots):
                if isinstance(r, torch.Tensor):
                    run = lambda: oned_graph_bfs_traverse_multi(g, bfs, r, p, with_depth=False)  # noqa: E731
                else:
                    run = lambda: oned_graph_bfs_traverse(g, bfs, r, p, with_depth=False)  # noqa: E731
                ms += _timed(run, lambda: oned_graph_bfs_reset(bfs, False, g))
        table.append((ms / reps, alpha, beta, blocks))
    best = min(table)
    return {"kind": "bfs", "alpha": best[1], "beta": best[2], "blocks": best[3], "ms": round(best[0], 4),
            "candidates": len(table)}


def tune_sssp(g: OnedGraph, roots, deltas=(0.08, 0.1, 0.2, 0.4), grids=None, pulls=(0.0, -1.0), subs=(0, -1),
              reps: int = 1) -> dict:
    """Best (delta, blocks, pull, sub_min) for SSSP over `roots` (a list: one
    search each; a device tensor: one multi-source search).  pull / sub_min
    are g5_sssp_params' heavy-phase pull threshold and sub-bucket threshold
    (0 = the library's default, -1 = off)."""
    st = SsspState(g)
    grids = _grids("sssp", g.nglobalverts) if grids is None else list(grids)
    table = []
    for delta, blocks, pull, sub in itertools.product(deltas, grids, pulls, subs):
        ms = 0.0
        for _ in range(reps):
            for r in _searches(roots):
                if isinstance(r, torch.Tensor):
                    run = lambda: oned_graph_sssp_traverse_multi(g, st, r, delta, blocks, pull, sub)  # noqa: E731
                else:
                    run = lambda: oned_graph_sssp_traverse(g, st, r, delta, blocks, pull, sub)  # noqa: E731
                ms += _timed(run, lambda: oned_graph_sssp_reset(st))
        table.append((ms / reps, delta, blocks, pull, sub))
    best = min(table)
    return {"kind": "sssp", "delta": best[1], "blocks": best[2], "pull": best[3], "sub_min": best[4],
            "ms": round(best[0], 4), "candidates": len(table)}


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
    return BfsParams(t["alpha"], t["beta"], 0, t["blocks"])


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
