#!/usr/bin/env python3
"""Graph500 BFS / SSSP benchmark on B200 (harmonic-mean GTEPS).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--scale S] [--impl ours|reference]

A step is one BFS from one Graph500 root (the runner's root choice,
examples/graph500_runner.cu:43-74) over the SCALE-S, edgefactor-16 Kronecker
graph generated and built into a CSR on the GPU beforehand.  `value` is the
harmonic-mean GTEPS of the K timed roots (nedge / time per root, nedge as the
reference's runner counts it), timed on the device with CUDA events;
between steps the working set (an 8.6 GB column array at SCALE 26) is far
larger than L2.  SSSP is timed the same way and reported under "sssp".

With N > 1 (torchrun, one rank per GPU) every rank holds its own copy of the
graph and takes every N-th root: weak scaling with no data-path collective;
`value` is all edges traversed / the slowest rank's time.

--impl reference times the reference algorithm's CPU implementation (the
reference has no CPU path of its own, so this is the oracle restatement in
oracle/) on all host cores, on the same workload, rank 0 only.
"""
from __future__ import annotations

import argparse
import gc
import importlib.util
import json
import os
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
PEAKS = os.path.join(REPO, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes (read + write) per traversed input edge of bfs_persistent_kernel on a
# main-component root, from an ncu capture at SCALE 23 (479.8 MB for 134,213,828 edges,
# with the bottom-up first-neighbour probe); scaled to the bench's roots by their edges.
TRAFFIC_BYTES_PER_EDGE = 3.57
E2E_REPS = 3  # end-to-end calls per root (median kept)
GATE_CYCLES = 200_000  # ~0.1 ms device-side spin queued before each timed root


def load_package():
    if "cgt_b200" in sys.modules:
        return sys.modules["cgt_b200"]
    pkg = os.path.join(REPO, "cuda-graph-traversal_b200")
    spec = importlib.util.spec_from_file_location("cgt_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cgt_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def metric_name(scale, ef):
    return f"harmonic-mean BFS GTEPS at SCALE {scale} ef{ef} (1 B200)"


def bench_config(scale, ef, K, world, csr_entries):
    """The workload, identical in both arms (ours and --impl reference)."""
    return {"workload": f"graph500 bfs scale{scale} ef{ef}", "scale": scale, "edgefactor": ef,
            "nverts": 1 << scale, "nedges": ef << scale, "csr_entries": int(csr_entries), "roots_per_rank": K,
            "roots": "runner root choice (seeds 2, 3): the K roots after the W warm-up roots",
            "l2": f"inputs larger than L2 (int32 column {csr_entries * 4 / 1e9:.1f} GB)",
            "parallelism": f"replicas x{world}, roots sharded"}


def hmean_gteps(nedge, secs):
    nedge = np.asarray(nedge, np.float64)
    secs = np.asarray(secs, np.float64)
    return float(1.0 / np.mean(secs / nedge) / 1e9)


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = os.path.join("/tmp", f"g5_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][1]) if rows[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def rank_roots(roots, rank, world):
    """Roots of one rank under weak scaling: every world-th root."""
    return roots[rank::world] or list(roots)


def combine_ranks(dist, device, total_ms, edges, hm):
    """Whole-job numbers: the slowest rank's time, all ranks' edges, and the
    sum of the ranks' harmonic means.  Every rank calls it (collectives)."""
    import torch
    t = torch.tensor([total_ms, edges, hm], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = t.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(sm[1]), float(sm[2])


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        pg = dist
    G = load_package()
    scale, ef = args.scale, args.edgefactor
    n, m = 1 << scale, ef << scale
    stream = torch.cuda.current_stream()

    # ---- setup (untimed): generation + CSR build on the GPU, as the runner.
    t0 = time.time()
    seed = G.make_mrg_seed(2, 3)
    ev0, ev1, ev2, ev3, ev4 = (torch.cuda.Event(enable_timing=True) for _ in range(5))
    ev0.record()
    tg = G.generate_kronecker_range(seed, scale, 0, m, device=dev)
    ev1.record()
    g = G.oned_graph_from_tuple_graph(tg, n, with_main=False, bfs_order=False, sssp_renumber=False)
    ev2.record()
    del tg
    G.oned_graph_bfs_order(g)  # the BFS's copy of the column, rows by decreasing neighbour degree
    ev3.record()
    G.oned_graph_sssp_renumber(g)  # the SSSP's copy in its own numbering, by decreasing degree
    ev4.record()
    torch.cuda.synchronize()
    gen_s, csr_s, order_s = ev0.elapsed_time(ev1) / 1e3, ev1.elapsed_time(ev2) / 1e3, ev2.elapsed_time(ev3) / 1e3
    renumber_s = ev3.elapsed_time(ev4) / 1e3
    t_main = time.perf_counter()
    g.main_bits = G.main_component_bitmap(g)  # one BFS from the hub: routes small-component roots
    main_s = time.perf_counter() - t_main
    torch.cuda.empty_cache()
    roots_all = G.generate_bfs_roots(g, 2, 3, 64)
    my_roots = rank_roots(roots_all, rank, world)
    K, W = args.steps, args.warmup
    seq = [my_roots[i % len(my_roots)] for i in range(W + K)]
    bfs = G.BfsState(g)
    # Roots outside the main component get a state of their own (the query
    # path routes them to the one-block search the same way), so the reset
    # before such a search undoes only the previous small search.
    bfs_s = G.BfsState(g)
    G.oned_graph_bfs_reset(bfs_s, with_depth=False, g=g)
    state = lambda r: bfs if g.in_main_component(r) else bfs_s  # noqa: E731
    vw = G._val_work(g)

    # Knobs of the main-component searches (alpha, beta and the work tiles
    # for BFS; the list tiles for SSSP at the reference's delta 0.1), tuned
    # on roots that are not timed (another root seed: 8 for BFS, 2 for SSSP)
    # or taken from the cache; the grid stays the library's (roots outside
    # the main component keep their one-block searches).
    tuned, bparams, skw = None, None, {}
    if not args.no_tune:
        import cgt_b200.autotune as T
        t_tune = time.time()
        cache = T.TuningCache(args.tune_cache)
        hits = (cache.get("bfs", g) is not None, cache.get("sssp", g) is not None)
        troots = [r for r in G.generate_bfs_roots(g, 5, 7, 64) if g.in_main_component(r)][:8]
        tb = cache.get("bfs", g) or T.tune_bfs(g, troots, alphas=(10.0, 14.0, 20.0), betas=(24.0,), grids=(0,), reps=2)
        ts = cache.get("sssp", g) or T.tune_sssp(g, troots[:2], deltas=(0.1,), grids=(0,), pulls=(0.0,), subs=(0,))
        if rank == 0:
            cache.put("bfs", g, tb)
            cache.put("sssp", g, ts)
        bparams = T.bfs_params(tb)
        skw = {"big_deg": ts["big_deg"], "chunk": ts["chunk"]}
        tuned = {"bfs": {k: tb[k] for k in ("alpha", "beta", "big_deg", "chunk", "lane_entries")},
                 "sssp": {k: ts[k] for k in ("delta", "big_deg", "chunk")}, "from_cache": list(hits),
                 "tune_s": round(time.time() - t_tune, 2), "tuning_roots": [int(r) for r in troots]}
    bp = lambda r: bparams if g.in_main_component(r) else None  # noqa: E731

    nedge, reached = {}, {}
    for r in set(seq):
        G.oned_graph_bfs_run(g, bfs, r, with_depth=False)
        st = G.bfs_stats(bfs)
        reached[r] = st.reached
        nedge[r] = G.edge_count(g, bfs.pred, vw)
    # Validate one tree per root set (untimed).
    r0 = seq[0]
    G.oned_graph_bfs_run(g, bfs, r0)
    dist = G.bfs_compute_dist_from_pred(g, bfs, r0)
    assert G.bfs_validate(g, r0, bfs.pred, dist, vw) == 0, "BFS validation failed"
    setup_s = time.time() - t0

    # Before each timed root the stream gets a short device-side spin, so the
    # reset and the search are both queued before the device reaches them:
    # the events then time the device work alone, not the host's launch of
    # the search behind a reset that finished in a microsecond.
    gate = lambda: torch.cuda._sleep(GATE_CYCLES)  # noqa: E731

    # ---- timed BFS.  The runner's protocol (examples/graph500_runner.cu:
    # 309-313): oned_graph_bfs_clear outside the timer, oned_graph_bfs_run
    # inside; here both run back to back on one stream and CUDA events split
    # them, so the reset time is reported too.
    for r in seq[:W]:
        G.oned_graph_bfs_reset(state(r), with_depth=False, g=g)
        G.oned_graph_bfs_traverse(g, state(r), r, bp(r), with_depth=False)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
            torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    with clocks:
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record()
        for i, r in enumerate(seq[W:]):
            a, b, c = evs[i]
            bs = state(r)
            gate()
            a.record()
            G.oned_graph_bfs_reset(bs, with_depth=False, g=g)
            b.record()
            G.oned_graph_bfs_traverse(g, bs, r, bp(r), with_depth=False)
            c.record()
        stop.record()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
    total_ms = start.elapsed_time(stop)
    step_s = [a.elapsed_time(c) / 1e3 for a, _, c in evs]
    kern_s = [b.elapsed_time(c) / 1e3 for _, b, c in evs]
    timed = seq[W:]
    t_nedge = [nedge[r] for r in timed]
    hm = hmean_gteps(t_nedge, kern_s)
    hm_with_reset = hmean_gteps(t_nedge, step_s)
    per_root_gteps = np.asarray(t_nedge, np.float64) / np.asarray(kern_s) / 1e9
    st = G.bfs_stats(state(timed[-1]))
    assert st.reached == reached[timed[-1]]
    big = [i for i, r in enumerate(timed) if nedge[r] >= 0.5 * max(t_nedge)]
    trace = G.bfs_trace(state(timed[-1]))

    # Roofline of the persistent BFS kernel over the roots in the big
    # component: algorithmic bytes per search = 2*nedge*4 (int32 col) +
    # reached*(8 rowstarts + 8 pred) (no depth array).
    alg_bytes = [2 * nedge[timed[i]] * 4 + reached[timed[i]] * 16 for i in big]
    achieved_gbs = float(np.sum(alg_bytes) / np.sum([kern_s[i] for i in big]) / 1e9)
    peak, peak_kind = hbm_peak()

    # ---- SSSP, same roots and protocol (a state of its own for roots
    # outside the main component, as for BFS).
    sssp, sssp_s = G.SsspState(g), G.SsspState(g)
    G.oned_graph_sssp_reset(sssp_s)
    sstate = lambda r: sssp if g.in_main_component(r) else sssp_s  # noqa: E731
    for r in seq[:W]:
        G.oned_graph_sssp_reset(sstate(r))
        G.oned_graph_sssp_traverse(g, sstate(r), r, **skw)
    sev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
            torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    torch.cuda.synchronize()
    nbuckets = nphases = 0
    s_validated = 0
    for i, r in enumerate(timed):
        ss = sstate(r)
        gate()
        sev[i][0].record()
        G.oned_graph_sssp_reset(ss)
        sev[i][1].record()
        G.oned_graph_sssp_traverse(g, ss, r, **skw)
        sev[i][2].record()
        # Every search's status is read (a device error -- a bounded wait
        # that expired, a list overflow -- raises) and its result validated
        # by the Graph500 SSSP rules; both run after the stop event.
        nbuckets, nphases = G.sssp_status(ss)
        assert G.sssp_validate(g, r, ss.dist, ss.pred, vw) == 0, f"SSSP validation failed for root {r}"
        s_validated += 1
    torch.cuda.synchronize()
    s_secs = [b.elapsed_time(c) / 1e3 for _, b, c in sev]
    s_secs_reset = [a.elapsed_time(c) / 1e3 for a, _, c in sev]
    s_hm = hmean_gteps(t_nedge, s_secs)
    s_per_root = np.asarray(t_nedge, np.float64) / np.asarray(s_secs) / 1e9
    s_alg_bytes = [2 * nedge[timed[i]] * 8 + reached[timed[i]] * 28 for i in big]
    s_achieved_gbs = float(np.sum(s_alg_bytes) / np.sum([s_secs[i] for i in big]) / 1e9)

    # ---- end to end through the C ABI with host buffers, the runner's
    # protocol: untimed clear, then per step the root goes host->device from
    # pinned memory, the search runs, and the step's result (its statistics:
    # levels and reached count) is read back to the host.
    # Each root's call is timed E2E_REPS times (reset untimed before each) and
    # its median kept: one host wall-clock sample of a ~10-50 us call is at the
    # mercy of host scheduling noise.
    e2e_s = []
    for r in timed:
        reps = []
        for _ in range(E2E_REPS):
            G.oned_graph_bfs_reset(state(r), with_depth=False, g=g)
            torch.cuda.synchronize()
            t = time.perf_counter()
            # one public call: the device reads the root from pinned host
            # memory, searches, and writes the statistics back to it
            res = G.oned_graph_bfs_query(g, state(r), int(r), params=bparams)
            reps.append(time.perf_counter() - t)
            assert res.reached == reached[r]
        e2e_s.append(float(np.median(reps)))
    e2e_hm = hmean_gteps(t_nedge, e2e_s)

    # The same calls with the search's result brought to the host as well:
    # right behind the search, g5_bfs_export's kernel writes one 16-byte
    # record (vertex, depth, parent) per reached vertex straight into pinned
    # host memory; one C call (g5_bfs_query_plan_export), one wait.
    xbuf = torch.empty(16 * n, dtype=torch.uint8).pin_memory()
    first_root = {}
    for r in timed:
        first_root.setdefault(id(state(r)), r)
    for r in first_root.values():  # each state's with-depth query plan made before timing
        G.oned_graph_bfs_reset(state(r), with_depth=True, g=g)
        G.oned_graph_bfs_query_export(g, state(r), int(r), with_depth=True, out=xbuf, params=bparams)
    e2e_res_s, e2e_res_bytes = [], []
    for r in timed:
        reps = []
        for _ in range(E2E_REPS):
            G.oned_graph_bfs_reset(state(r), with_depth=True, g=g)
            torch.cuda.synchronize()
            t = time.perf_counter()
            _, rec = G.oned_graph_bfs_query_export(g, state(r), int(r), with_depth=True, out=xbuf, params=bparams)
            reps.append(time.perf_counter() - t)
            assert len(rec) == reached[r]
        root_rec = rec[rec["vertex"] == r]
        assert len(root_rec) == 1 and root_rec["parent"][0] == r and root_rec["depth"][0] == 0
        e2e_res_s.append(float(np.median(reps)))
        e2e_res_bytes.append(24 + 8 + 16 * len(rec))
    e2e_res_hm = hmean_gteps(t_nedge, e2e_res_s)
    del xbuf

    # Whole-job numbers across ranks: slowest rank's time, all ranks' edges.
    tot_edges = float(np.sum(t_nedge))
    max_ms = total_ms
    # Per rank the Graph500 harmonic mean; across ranks (weak scaling) the
    # ranks' harmonic means add up.
    value = hm
    if pg:
        max_ms, tot_edges, value = combine_ranks(pg, dev, total_ms, tot_edges, hm)

    # ---- CPU baseline (rank 0, one GPU): the oracle's top-down BFS on the
    # host cores over the same timed roots; each root's depth array is also
    # compared with the GPU's (the parity check at this scale).
    cpu = None
    parity = {"sssp_validated": s_validated, "bfs_trees_validated": 1}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        def gpu_depth(r):
            # the GPU's depth array for r, its parent tree validated on the way
            G.oned_graph_bfs_run(g, bfs, r)
            d = G.bfs_compute_dist_from_pred(g, bfs, r)
            assert G.bfs_validate(g, r, bfs.pred, d, vw) == 0, f"BFS validation failed for root {r}"
            parity["bfs_trees_validated"] += 1
            return bfs.depth.cpu().numpy()
        cpu_roots = timed if args.cpu_roots <= 0 else timed[:args.cpu_roots]
        cpu, checked = cpu_baseline_sample(g, cpu_roots, nedge, gpu_depth)
        parity[f"s{scale}_depth_roots_checked"] = checked
    if rank == 0:
        line = {
            "metric": metric_name(scale, ef),
            "value": float(f"{value:.6g}"),
            "unit": "GTEPS",
            "n_gpus": world,
            "steps": K,
            "warmup": W,
            "ms_per_step": round(max_ms / K, 4),
            "timing": "device events per root (queued behind a 0.1 ms device spin, so host launch latency stays "
                      "out); reset (the runner's oned_graph_bfs_clear) untimed as in the runner",
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int32",
            "data": "synthetic: Graph500 Kronecker generator (A,B,C,D = .57,.19,.19,.05), seeds (2,3), bit-identical to the reference's",
            "config": bench_config(scale, ef, K, world, g.nlocaledges),
            "aggregate_gteps": round(tot_edges / (max_ms / 1e3) / 1e9, 3),
            "hmean_gteps_with_reset": float(f"{hm_with_reset:.6g}"),
            "median_gteps": round(float(np.median(per_root_gteps)), 3),
            "small_component_roots": int(sum(1 for r in timed if nedge[r] < 0.5 * max(t_nedge))),
            "small_root_us_max": round(max([kern_s[i] for i, r in enumerate(timed) if nedge[r] < 0.5 * max(t_nedge)]
                                           or [0.0]) * 1e6, 2),
            "big_root_ms_mean": round(float(np.mean([kern_s[i] for i in big])) * 1e3, 4),
            "trace_last_root": trace,
            "roofline": {"bound": "hbm", "kernel": "bfs_persistent_kernel",
                         "achieved": round(achieved_gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved_gbs / peak, 4), "peak_kind": f"{peak_kind} copy bandwidth",
                         "bytes_per_launch": int(np.mean(alg_bytes)),
                         "bytes_model": "2*nedge*4 (col) + reached*(8 rowstarts + 8 pred)",
                         "kernel_ms_mean": round(float(np.mean(kern_s)) * 1e3, 4),
                         "traffic": int(args.traffic if args.traffic is not None
                                        else TRAFFIC_BYTES_PER_EDGE * np.mean([nedge[timed[i]] for i in big])),
                         "traffic_source": "ncu dram__bytes_read+write given by --traffic" if args.traffic
                         is not None else "ncu capture at SCALE 23: 3.57 B per traversed edge, scaled by edges"},
            "e2e": {"value": float(f"{(e2e_hm if world == 1 else e2e_hm * world):.6g}"), "unit": "GTEPS",
                    "h2d_bytes_per_step": 8, "d2h_bytes_per_step": 24,
                    "small_root_us": round(min(e2e_s) * 1e6, 1) if e2e_s else None,
                    "timing": f"median of {E2E_REPS} calls per root (reset untimed before each)",
                    "path": "oned_graph_bfs_query -> C ABI g5_bfs_query after an untimed reset: the kernel "
                            "reads the 8-byte root from pinned host memory and writes the 24-byte stats back "
                            "to pinned host memory (over PCIe, inside the timed call), host wall clock",
                    "with_result": {
                        "value": float(f"{(e2e_res_hm if world == 1 else e2e_res_hm * world):.6g}"),
                        "unit": "GTEPS", "h2d_bytes_per_step": 8,
                        "d2h_bytes_per_step": int(np.mean(e2e_res_bytes)) if e2e_res_bytes else 0,
                        "small_root_us": round(min(e2e_res_s) * 1e6, 1) if e2e_res_s else None,
                        "big_root_ms_mean": round(float(np.mean([e2e_res_s[i] for i in big])) * 1e3, 3)
                        if big else None,
                        "path": "oned_graph_bfs_query_export -> C ABI g5_bfs_query_plan_export after an "
                                "untimed reset: the search, then one 16-byte record (vertex, depth, parent) per "
                                "reached vertex written by a kernel into pinned host memory, one host wait, "
                                "median of 3 calls per root"}},
            "sssp": {"value": float(f"{s_hm:.6g}"), "unit": "GTEPS (harmonic mean)",
                     "hmean_gteps_with_reset": float(f"{hmean_gteps(t_nedge, s_secs_reset):.6g}"),
                     "median_gteps": round(float(np.median(s_per_root)), 3),
                     "big_root_ms_mean": round(float(np.mean([s_secs[i] for i in big])) * 1e3, 3),
                     "buckets_last_root": nbuckets, "phases_last_root": nphases, "delta": 0.1,
                     "validated": s_validated,
                     # The SSSP kernel against the same HBM roofline: algorithmic bytes
                     # per search = 2*nedge*(4 col + 4 w) + reached*(8 rowstarts + 8
                     # packed distance/parent + 12 output).
                     "roofline": {"bound": "hbm", "kernel": "sssp_persistent_kernel",
                                  "achieved": round(s_achieved_gbs, 1), "peak": peak, "unit": "GB/s",
                                  "frac": round(s_achieved_gbs / peak, 4),
                                  "bytes_per_launch": int(np.mean(s_alg_bytes)),
                                  "bytes_model": "2*nedge*8 (col + w) + reached*(8 rowstarts + 8 packed + 12 out)"}},
            "construction": {"generation_s": round(gen_s, 4), "csr_build_s": round(csr_s, 4),
                             "bfs_degree_order_s": round(order_s, 4), "sssp_renumber_s": round(renumber_s, 4),
                             "main_component_s": round(main_s, 4), "setup_total_s": round(setup_s, 2),
                             "note": "device events; the CSR build includes its first-use allocations"},
            "nedge_per_root": int(np.median(t_nedge)),
            "clocks": clocks.summary(),
            "gpu_launches": K,
            "gpu_launches_note": "one bfs_persistent_kernel per step (+ memsets); SSSP timed separately",
        }
        if cpu:
            line["cpu_baseline"] = cpu
        line["parity"] = parity
        line["autotuned"] = tuned
        if world == 1:
            # The SCALE-26 graph is not needed any more: drop it and every
            # closure that holds it, so the later legs get the memory.
            del g, bfs, bfs_s, vw, sssp, sssp_s, state, sstate, bp, bs, ss
            if cpu:
                del gpu_depth
            gc.collect()
            torch.cuda.empty_cache()
            line["memory_after_free_gb"] = round(torch.cuda.memory_allocated() / 1e9, 2)
        if world == 1 and not args.no_reference_gpu:
            line["reference_gpu"] = run_reference_gpu(scale, ef, roots_all, W, K, nedge, kern_s, s_secs, e2e_s)
        if world == 1 and not args.no_batched:
            line["batched"] = run_batched(G, dev, args.batched_scale, args.edgefactor, args.batched_roots)
            torch.cuda.empty_cache()
        if world == 1 and not args.no_batched:
            line["sssp_batched"] = run_sssp_batched(G, dev, args.sssp_batched_scale, args.edgefactor)
            torch.cuda.empty_cache()
        if world == 1 and not args.no_packed:
            line["packed"] = run_packed(G, dev, args.packed_graphs, args.packed_min_scale, args.packed_max_scale,
                                        args.edgefactor)
            torch.cuda.empty_cache()
        if world == 1 and not args.no_serve:
            line["serving"] = run_serving(G, dev, args.serve_queries, args.serve_rate, args.edgefactor, args.serve_slots,
                                          args.serve_low_rate, not args.serve_count_errors)
        line["headline"] = headline(line)
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def run_batched(G, dev, scale, ef, nroots, reps=3):
    """Batched BFS: `nroots` Graph500 roots (the runner's root choice) in
    one g5_msbfs search on the SCALE-`scale` Kronecker graph, against the
    same roots searched one by one with the single-root BFS.  Aggregate
    GTEPS = sum of the roots' TEPS edge counts / device time.  The batch's
    depth arrays are compared with the single searches' for every 16th root."""
    import torch
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    t0 = time.time()
    g = G.oned_graph_from_kronecker(G.make_mrg_seed(2, 3), scale, ef << scale, device=dev)
    roots = G.generate_bfs_roots(g, 2, 3, nroots)
    a, b = ev(), ev()
    a.record()
    ms = G.MsBfsState(g)
    b.record()
    torch.cuda.synchronize()
    prep_ms = a.elapsed_time(b)
    depth8 = torch.empty((len(roots), g.nglobalverts), dtype=torch.uint8, device=dev)
    import cgt_b200.autotune as T
    tuned = T.tune_msbfs(g, roots, alphas=(16.0, 32.0, 64.0), checks=(0, 2), ms=ms)
    params = T.msbfs_params(tuned)
    G.msbfs_run(g, ms, roots, params)  # warm-up
    search_ms, full_ms = [], []
    for _ in range(reps):
        a, b, c = ev(), ev(), ev()
        a.record()
        G.msbfs_run(g, ms, roots, params, sync=False)
        b.record()
        G.msbfs_depths_u8(ms, depth8)
        c.record()
        torch.cuda.synchronize()
        search_ms.append(a.elapsed_time(b))
        full_ms.append(a.elapsed_time(c))
    st = G.msbfs_stats(ms)
    trace = G.msbfs_trace(ms)
    # The same roots one at a time (reset untimed, as the runner's clear).
    bfs = G.BfsState(g)
    vw = G._val_work(g)
    plain_ms, nedge, checked = 0.0, [], 0
    for i, r in enumerate(roots):
        G.oned_graph_bfs_reset(bfs, True, g)
        a, b = ev(), ev()
        a.record()
        G.oned_graph_bfs_traverse(g, bfs, r, None, True)
        b.record()
        torch.cuda.synchronize()
        plain_ms += a.elapsed_time(b)
        nedge.append(G.edge_count(g, bfs.pred, vw))
        if i % 16 == 0:
            want = bfs.depth.to(torch.int64)
            got = depth8[i].to(torch.int64)
            got[got == 255] = -1
            assert torch.equal(want, got), f"batched depth of root {r} differs from the single search"
            checked += 1
    E = float(sum(nedge))
    best, best_full = min(search_ms), min(full_ms)
    return {"workload": f"multi-source bfs scale{scale} ef{ef}, {len(roots)} roots in one search",
            "value": round(E / best / 1e6, 1), "unit": "GTEPS (aggregate over the batch)",
            "ms_per_batch": round(best, 3), "ms_per_batch_with_depth_export": round(best_full, 3),
            "plain_ms_total": round(plain_ms, 3), "plain_gteps": round(E / plain_ms / 1e6, 1),
            "speedup_vs_plain": round(plain_ms / best, 2),
            "speedup_vs_plain_with_export": round(plain_ms / best_full, 2),
            "depth_arrays_checked_identical": checked, "levels": st.levels, "pull_levels": st.pull_levels,
            "level_ms": [round(x, 3) for x in trace["ms"]], "level_mode": trace["mode"],
            "prepare_ms": round(prep_ms, 2), "setup_s": round(time.time() - t0, 2),
            "autotuned": {k: tuned[k] for k in ("alpha", "check_frontier", "blocks", "candidates")},
            "timing": "device events, min of 3 after one warm-up; plain = single-root traverse with depth, "
                      "reset untimed"}


def run_sssp_batched(G, dev, scale, ef, nsources=32, reps=3):
    """Batched SSSP: `nsources` Graph500 roots of the SCALE-`scale` Kronecker
    graph in one g5_sssp_multi_run, against the same sources one at a time
    with the single-source search (reset untimed).  Every source's distance
    and parent arrays are compared bit for bit; aggregate GTEPS = sum of the
    sources' TEPS edge counts / device time."""
    import torch
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    t0 = time.time()
    g = G.oned_graph_from_kronecker(G.make_mrg_seed(2, 3), scale, ef << scale, device=dev)
    roots = G.generate_bfs_roots(g, 2, 3, nsources)
    work = G.sssp_multi_workspace(g)
    G.oned_graph_sssp_multi(g, roots, work=work)  # warm-up
    times = []
    for _ in range(reps):
        a, b = ev(), ev()
        a.record()
        dist, pred, st = G.oned_graph_sssp_multi(g, roots, work=work)
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    ss = G.SsspState(g)
    vw = G._val_work(g)
    plain_ms, nedge, checked = 0.0, [], 0
    for i, r in enumerate(roots):
        G.oned_graph_sssp_reset(ss)
        torch.cuda.synchronize()
        a, b = ev(), ev()
        a.record()
        G.oned_graph_sssp_traverse(g, ss, int(r))
        b.record()
        torch.cuda.synchronize()
        G.sssp_status(ss)
        plain_ms += a.elapsed_time(b)
        assert torch.equal(dist[i].view(torch.int32), ss.dist.view(torch.int32)) and torch.equal(pred[i], ss.pred), \
            f"batched SSSP of source {r} differs from the single-source search"
        checked += 1
        nedge.append(G.edge_count(g, ss.pred, vw))
    assert G.sssp_validate(g, int(roots[0]), dist[0], pred[0], vw) == 0
    E = float(sum(nedge))
    best = min(times)
    return {"workload": f"batched sssp scale{scale} ef{ef}, {len(roots)} sources in one launch",
            "value": round(E / best / 1e6, 2), "unit": "GTEPS (aggregate over the batch)",
            "ms_per_batch": round(best, 3), "plain_ms_total": round(plain_ms, 3),
            "plain_gteps": round(E / plain_ms / 1e6, 2), "speedup_vs_plain": round(plain_ms / best, 2),
            "sources_checked_identical": checked, "rounds": st.rounds,
            "entries_scanned_per_entry": round(st.entries_scanned / max(1, g.nlocaledges), 2),
            "setup_s": round(time.time() - t0, 2),
            "timing": "device events, min of 3 after one warm-up; plain = single-source traverse, reset untimed",
            "note": "a win up to about 2^20 vertices (SCALE 14: 10-13x, 18: 3.6-3.9x, 20: 1.5-1.7x); from SCALE 22 "
                    "the single-source delta-stepping search is faster (0.7x at 22, 0.27x at 26)"}


def run_packed(G, dev, ngraphs, smin, smax, ef, reps=3):
    """Many small graphs: `ngraphs` Kronecker graphs with SCALE drawn
    uniformly from [smin, smax] (seeded), one BFS and one SSSP root each (the
    graph's first Graph500 root), packed into one CSR and run as one CUDA
    graph (reset, multi-root BFS, reset, multi-source SSSP).  Baseline: the
    same graphs one at a time, each a plain g5_bfs_run + g5_sssp_run on its
    own CSR.  Aggregate GTEPS = sum of the graphs' TEPS edge counts / time."""
    import torch
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    rng = np.random.default_rng(2024)
    scales = rng.integers(smin, smax + 1, size=ngraphs).tolist()
    t0 = time.time()
    pk = G.pack_kronecker(scales, edgefactor=ef, seed1_base=100, seed2=3, device=dev)
    import cgt_b200.autotune as T
    tb = T.tune_bfs(pk.g, pk.d_roots, alphas=(10.0, 14.0, 20.0), betas=(24.0,), grids=(0,))
    ts = T.tune_sssp(pk.g, pk.d_roots, deltas=(0.08, 0.1, 0.2, 0.4), grids=(0,))
    batch = G.PackedBatch(pk, delta=ts["delta"], capture=True, bfs_params=T.bfs_params(tb),
                          sssp_blocks=ts["blocks"], sssp_pull=ts["pull"], sssp_sub_min=ts["sub_min"],
                          sssp_big_deg=ts["big_deg"], sssp_chunk=ts["chunk"])
    build_s = time.time() - t0
    bfs_ms, all_ms = [], []
    for _ in range(reps):
        a, b, c = ev(), ev(), ev()
        a.record(batch.stream)
        batch.run()
        c.record(batch.stream)
        torch.cuda.synchronize()
        all_ms.append(a.elapsed_time(c))
    batch.check()
    # BFS alone (eager, same stream), for the BFS share.
    for _ in range(reps):
        a, b = ev(), ev()
        with torch.cuda.stream(batch.stream):
            G.oned_graph_bfs_reset(batch.bfs, True, pk.g)
            a.record(batch.stream)
            G.oned_graph_bfs_traverse_multi(pk.g, batch.bfs, pk.d_roots, batch.bfs_params)
            b.record(batch.stream)
        torch.cuda.synchronize()
        bfs_ms.append(a.elapsed_time(b))
    vw = G._val_work(pk.g)
    nedge = G.edge_count(pk.g, batch.bfs.pred, vw)  # sum of every graph's TEPS edge count
    depth = batch.bfs.depth.cpu().numpy()
    dist = batch.sssp.dist.cpu().numpy()
    del batch, vw
    torch.cuda.empty_cache()
    # One at a time: each graph rebuilt on its own, plain BFS + SSSP timed.
    plain_bfs, plain_sssp, checked = 0.0, 0.0, 0
    for i, s in enumerate(scales):
        g = G.oned_graph_from_kronecker(G.make_mrg_seed(100 + i, 3), s, ef << s, device=dev, with_main=False)
        r = int(pk.local_roots[i])
        bfs, ss = G.BfsState(g), G.SsspState(g)
        a, b, c = ev(), ev(), ev()
        a.record()
        G.oned_graph_bfs_run(g, bfs, r)
        b.record()
        G.oned_graph_sssp_run(g, ss, r, delta=ts["delta"])
        c.record()
        torch.cuda.synchronize()
        plain_bfs += a.elapsed_time(b)
        plain_sssp += b.elapsed_time(c)
        if i % 50 == 0:
            sl = pk.graph_slice(i)
            assert np.array_equal(depth[sl], bfs.depth.cpu().numpy()), f"packed BFS of graph {i} differs"
            assert np.array_equal(dist[sl].view(np.uint32), ss.dist.cpu().numpy().view(np.uint32)), \
                f"packed SSSP of graph {i} differs"
            checked += 1
    best, best_bfs = min(all_ms), min(bfs_ms)
    return {"workload": f"{ngraphs} Kronecker graphs, SCALE uniform in [{smin}, {smax}], ef{ef}, "
                        "one BFS + one SSSP root each, packed into one CSR, one CUDA graph per batch",
            "vertices": int(pk.g.nglobalverts), "csr_entries": int(pk.g.nlocaledges),
            "ms_per_batch": round(best, 3), "bfs_ms": round(best_bfs, 3),
            "bfs_gteps": round(nedge / best_bfs / 1e6, 2),
            "bfs_plus_sssp_gteps": round(2 * nedge / best / 1e6, 2),
            "plain_ms_total": round(plain_bfs + plain_sssp, 2), "plain_bfs_ms": round(plain_bfs, 2),
            "plain_sssp_ms": round(plain_sssp, 2),
            "speedup_vs_plain": round((plain_bfs + plain_sssp) / best, 2),
            "bfs_speedup_vs_plain": round(plain_bfs / best_bfs, 2),
            "graphs_checked_identical": checked, "build_s": round(build_s, 2),
            "autotuned": {"bfs_alpha": tb["alpha"], "bfs_beta": tb["beta"], "bfs_big_deg": tb["big_deg"],
                          "bfs_chunk": tb["chunk"], "bfs_lane_entries": tb["lane_entries"],
                          "sssp_delta": ts["delta"], "sssp_pull": ts["pull"], "sssp_sub_min": ts["sub_min"],
                          "sssp_big_deg": ts["big_deg"], "sssp_chunk": ts["chunk"]},
            "timing": "device events; batch = replay of the captured CUDA graph (BFS+SSSP resets included), "
                      "min of 3 after a warm-up; plain = per-graph g5_bfs_run + g5_sssp_run, resets included"}


SERVE_SCALES = (16, 18, 20, 22, 22, 23, 24, 24)


def run_serving(G, dev, nqueries, rate, ef=16, slots=8, low_rate=250.0, raise_errors=True):
    """Serving: 8 resident Kronecker graphs (SCALE 16, 18, 20, 22, 22, 23, 24,
    24; seeds (2+i, 3)), a Poisson stream of queries (70% BFS, 30% SSSP,
    uniform graph, uniform non-zero-degree root, seed 1) replayed in real
    time through the continuous-batching server, then through plain calls
    one query at a time.  Latency = completion seen by the host - arrival.
    `rate` saturates both (throughput); a second trace at `low_rate`, below
    the server's capacity, shows latency when queries do not pile up."""
    import torch
    import cgt_b200.serve as S
    t0 = time.time()
    graphs = [G.oned_graph_from_kronecker(G.make_mrg_seed(2 + i, 3), s, ef << s, device=dev, with_main=False)
              for i, s in enumerate(SERVE_SCALES)]
    build_s = time.time() - t0
    trace = S.poisson_trace(graphs, nqueries, rate, bfs_share=0.7, seed=1)
    warm = S.poisson_trace(graphs, 64, rate, bfs_share=0.5, seed=99)
    srv = S.GraphServer(graphs, slots=slots, hbm_reserve=16 << 30, max_sssp_per_graph=slots, raise_errors=raise_errors)
    srv.prewarm()  # workspaces created up front (admission by free HBM)
    srv.run_trace(warm, deadline=600)  # batched copies prepared, kernels loaded
    srv.stats = S.ServerStats()
    res = srv.run_trace(trace, deadline=3600)
    ours = S.latency_summary(res)
    st = srv.stats
    del srv
    torch.cuda.empty_cache()
    low = None
    if low_rate:
        ltrace = S.poisson_trace(graphs, nqueries, low_rate, bfs_share=0.7, seed=2)
        srv = S.GraphServer(graphs, slots=slots, hbm_reserve=16 << 30, max_sssp_per_graph=slots, raise_errors=raise_errors)
        srv.prewarm()
        srv.run_trace(warm, deadline=600)
        srv.stats = S.ServerStats()
        low = {"rate_qps": low_rate, "ours": S.latency_summary(srv.run_trace(ltrace, deadline=3600)),
               "device_errors": srv.stats.device_errors, "errors": srv.stats.errors}
        del srv
        torch.cuda.empty_cache()
    S.serve_plain(graphs, warm)
    plain = S.latency_summary(S.serve_plain(graphs, trace))
    if low:
        low["plain_one_at_a_time"] = S.latency_summary(S.serve_plain(graphs, ltrace))
    kinds = {k: S.latency_summary([r for r in res if r.kind == k]) for k in ("bfs", "sssp")}
    return {"workload": f"{len(graphs)} resident graphs SCALE {list(SERVE_SCALES)} ef{ef}, {nqueries} Poisson "
                        f"queries at {rate:g}/s (70% BFS, 30% SSSP)",
            "qps": ours["qps"], "p50_ms": ours["p50_ms"], "p99_ms": ours["p99_ms"],
            "makespan_s": ours["makespan_s"], "by_kind": kinds,
            "plain_one_at_a_time": plain, "qps_vs_plain": round(ours["qps"] / plain["qps"], 2),
            "bfs_batches": st.bfs_batches, "bfs_queries_batched": st.bfs_batched_queries,
            "sssp_launches": st.sssp_launches, "sssp_batches": st.sssp_batches,
            "sssp_queries_batched": st.sssp_batched_queries, "max_concurrent_launches": st.max_inflight,
            "device_errors": st.device_errors, "errors": st.errors,
            "slots": slots, "low_load": low, "build_s": round(build_s, 2),
            "timing": "host clock: latency from a query's arrival time to the host seeing its launch's "
                      "CUDA event complete; BFS results exported as depth arrays"}


def run_kernels_once(scale, ef):
    """Every kernel of the path once, through the public API, checked: the
    command that the per-kernel ncu summaries capture."""
    import torch
    G = load_package()
    torch.cuda.set_device(0)
    seed = G.make_mrg_seed(2, 3)
    tg = G.generate_kronecker_range(seed, scale, 0, ef << scale)  # kron_generate_kernel
    g = G.oned_graph_from_tuple_graph(tg, 1 << scale)  # count, partition, place, row sorts, split, degree order
    del tg
    r = next(x for x in G.generate_bfs_roots(g, 2, 3, 8) if g.in_main_component(x))
    bfs, vw = G.BfsState(g), G._val_work(g)
    G.oned_graph_bfs_run(g, bfs, r)
    d = G.bfs_compute_dist_from_pred(g, bfs, r)
    ne = G.edge_count(g, bfs.pred, vw)  # edge_count_kernel
    rec = G.oned_graph_bfs_export(g, bfs)  # bfs_export_kernel (a grid search's result: a scan of the parents)
    assert len(rec) == G.bfs_stats(bfs).reached
    err = G.bfs_validate(g, r, bfs.pred, d, vw)  # bfs_val_edge_kernel
    s = G.SsspState(g)
    G.oned_graph_sssp_run(g, s, r)
    G.sssp_status(s)
    serr = G.sssp_validate(g, r, s.dist, s.pred, vw)  # sssp_val_edge_kernel
    roots32 = [x for x in G.generate_bfs_roots(g, 2, 3, 64) if g.in_main_component(x)][:32]
    md, _, _ = G.oned_graph_sssp_multi(g, roots32, with_pred=False)  # mss_persistent_kernel
    assert torch.equal(md[roots32.index(r)].view(torch.int32), s.dist.view(torch.int32)) if r in roots32 else True
    torch.cuda.synchronize()
    print(json.dumps({"scale": scale, "root": int(r), "nedge": int(ne), "bfs_errors": int(err),
                      "sssp_errors": int(serr)}), flush=True)
    if err or serr:
        raise SystemExit("validation failed")


def run_batched_only(args):
    import torch
    torch.cuda.set_device(0)
    G = load_package()
    dev = torch.device("cuda", 0)
    out = {}
    if args.only_batched in ("msbfs", "all"):
        out["batched"] = run_batched(G, dev, args.batched_scale, args.edgefactor, args.batched_roots)
    if args.only_batched in ("sssp", "all"):
        out["sssp_batched"] = run_sssp_batched(G, dev, args.sssp_batched_scale, args.edgefactor)
    if args.only_batched in ("packed", "all"):
        out["packed"] = run_packed(G, dev, args.packed_graphs, args.packed_min_scale, args.packed_max_scale,
                                   args.edgefactor)
    if args.only_batched in ("serve", "all"):
        out["serving"] = run_serving(G, dev, args.serve_queries, args.serve_rate, args.edgefactor, args.serve_slots,
                                     args.serve_low_rate, not args.serve_count_errors)
    print(json.dumps(out), flush=True)


def cpu_baseline_sample(g, roots, nedge, gpu_depth=None):
    """Oracle BFS (the reference's top-down algorithm, OpenMP on all host
    cores) on the same CSR, copied to the host, for `roots` (the timed roots:
    the same harmonic mean as `value`).  With gpu_depth(r) -> the GPU's
    depth array for root r, every root's oracle depth array is compared with
    it (a mismatch raises).  Returns (baseline dict, roots compared)."""
    from oracle import oracle as O
    rs = g.rowstarts.cpu().numpy().view(np.uint64)
    col = g.col.cpu().numpy().view(np.uint32)
    n = g.nglobalverts
    pred = np.empty(n, np.int64)
    depth = np.empty(n, np.int64)
    secs, checked, seen = [], 0, set()
    for r in roots:
        O.bfs_clear(n, pred, depth)
        t = time.perf_counter()
        O.bfs_search(rs, col, n, r, pred, depth)
        secs.append(time.perf_counter() - t)
        if gpu_depth is not None and r not in seen:
            seen.add(r)
            got = gpu_depth(r)
            if not np.array_equal(got.astype(np.int64), depth):
                raise AssertionError(f"GPU depth array of root {r} differs from the oracle's "
                                     f"({int(np.count_nonzero(got.astype(np.int64) != depth))} vertices)")
            checked += 1
    ne = np.asarray([nedge[r] for r in roots], np.float64)
    big = ne >= 0.5 * ne.max()
    out = {"value": float(f"{hmean_gteps(ne, secs):.6g}"), "unit": "GTEPS",
           "cores": O.num_threads(), "kind": "port",
           "median_gteps": round(float(np.median(ne / np.asarray(secs) / 1e9)), 4),
           "big_root_median_gteps": round(float(np.median((ne / np.asarray(secs) / 1e9)[big])), 4),
           "sample": f"the {len(roots)} timed roots of the same graph (the harmonic mean of `value`), oracle "
                     "top-down BFS (OpenMP), clear untimed as in the runner"}
    return out, checked


REF_BENCH = os.path.join(REPO, "oracle", "_ref", "ref_bench")


def run_reference_gpu(scale, ef, roots, W, K, nedge, bfs_secs, sssp_secs, e2e_secs, sssp_big=2):
    """The reference itself (its library built from its own sources into
    oracle/_ref/ref_bench by oracle/ref.mk, np=1 through the single-process
    shims) on this GPU, with its runner's protocol and host wall clock: BFS
    from the same K timed roots, SSSP from the timed roots outside the main
    component plus the first `sssp_big` main-component ones (a reference
    SSSP of the big component takes ~5 s).  TEPS edge counts are this
    graph's (the same graph, roots and counting rule)."""
    if not os.path.exists(REF_BENCH):
        return {"unavailable": "oracle/_ref/ref_bench is not built (the reference sources were absent at build)"}
    timed = [roots[(W + i) % len(roots)] for i in range(K)]
    t_ne = np.asarray([nedge[r] for r in timed], np.float64)
    big = [i for i in range(K) if t_ne[i] >= 0.5 * t_ne.max()]
    small = [i for i in range(K) if i not in big]
    s_idx = sorted(set(small + big[:sssp_big]))
    s_abs = [(W + i) % len(roots) for i in s_idx]
    cmd = [REF_BENCH, str(scale), str(ef), str(K), "0", str(W), "0"] + [str(j) for j in s_abs]
    t0 = time.time()
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=900, check=True).stdout
        rb = json.loads(out.strip().splitlines()[-1])
    except Exception as ex:  # noqa: BLE001 -- a missing or failing reference is reported, not fatal
        return {"unavailable": f"ref_bench failed: {str(ex)[:200]}"}
    b_root = [int(x[0]) for x in rb["bfs"]]
    assert b_root == timed, "reference roots differ from ours"
    b_t = np.asarray([float(x[1]) for x in rb["bfs"]])
    s_t = {int(x[0]): float(x[1]) for x in rb["sssp"]}
    ours_b = np.asarray(bfs_secs)
    res = {"what": "the reference's own library (np=1, built from its sources), same graph and roots, "
                   "host wall clock around each synchronous oned_graph_*_run as its runner times it",
           "generation_s": round(rb["generation_s"], 3), "construction_s": round(rb["construction_s"], 3),
           "bfs": {"value": float(f"{hmean_gteps(t_ne, b_t):.6g}"), "unit": "GTEPS (harmonic mean, same K roots)",
                   "median_gteps": round(float(np.median(t_ne / b_t / 1e9)), 4),
                   "big_root_ms_median": round(float(np.median(b_t[big])) * 1e3, 3),
                   "small_root_us": round(float(np.min(b_t[small])) * 1e6, 1) if small else None},
           "sssp": {"roots": [timed[i] for i in s_idx], "ms": [round(s_t[timed[i]] * 1e3, 3) for i in s_idx],
                    "big_root_ms_median": round(float(np.median([s_t[timed[i]] for i in big[:sssp_big]])) * 1e3, 1),
                    "small_root_ms": round(min(s_t[timed[i]] for i in small) * 1e3, 3) if small else None},
           "run_s": round(time.time() - t0, 1)}
    ours_s = np.asarray(sssp_secs)
    ref_s_big = np.median([s_t[timed[i]] for i in big[:sssp_big]])
    res["ours_over_reference"] = {
        "bfs_hmean": round(hmean_gteps(t_ne, ours_b) / res["bfs"]["value"], 2),
        "bfs_hmean_e2e": round(hmean_gteps(t_ne, e2e_secs) / res["bfs"]["value"], 2),
        "bfs_big_root_median": round(float(np.median(b_t[big]) / np.median(ours_b[big])), 1),
        "sssp_big_root_median": round(float(ref_s_big / np.median(ours_s[big])), 1),
        "sssp_small_root": round(float(min(s_t[timed[i]] for i in small) / np.min(ours_s[small])), 1)
        if small else None}
    return res


def headline(line):
    """A compact summary placed last in the line."""
    h = {"bfs_hmean_gteps": line["value"], "bfs_median_gteps": line.get("median_gteps"),
         "bfs_roofline_frac": line["roofline"]["frac"], "e2e_hmean_gteps": line["e2e"]["value"],
         "sssp_hmean_gteps": line["sssp"]["value"], "sssp_median_gteps": line["sssp"]["median_gteps"],
         "sssp_roofline_frac": line["sssp"]["roofline"]["frac"], "parity": line.get("parity")}
    t = line.get("autotuned")
    if t:
        h["tuned"] = {"bfs": t["bfs"], "sssp": t["sssp"]}
    if "cpu_baseline" in line:
        h["cpu_hmean_gteps"] = line["cpu_baseline"]["value"]
    rg = line.get("reference_gpu")
    if rg and "bfs" in rg:
        h["reference_gpu_bfs_hmean_gteps"] = rg["bfs"]["value"]
        h["ours_over_reference_gpu"] = rg["ours_over_reference"]
    if "batched" in line:
        h["batched_256_speedup"] = line["batched"]["speedup_vs_plain"]
    if "sssp_batched" in line:
        h["sssp_batched_32_speedup"] = line["sssp_batched"]["speedup_vs_plain"]
    if "packed" in line:
        h["packed_speedup"] = line["packed"]["speedup_vs_plain"]
    if "serving" in line:
        sv = line["serving"]
        h["serving"] = {"qps": sv["qps"], "p50_ms": sv["p50_ms"], "p99_ms": sv["p99_ms"],
                        "qps_vs_plain": sv["qps_vs_plain"], "device_errors": sv["device_errors"]}
    return h


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    from oracle import oracle as O
    scale, ef = args.scale, args.edgefactor
    n, m = 1 << scale, ef << scale
    t0 = time.time()
    seed = O.make_mrg_seed(2, 3)
    e, w = O.generate_kronecker_range(seed, scale, 0, m)
    gen_s = time.time() - t0
    t1 = time.time()
    rs, col, cw = O.csr_build(e, w, n, canonical=False)
    csr_s = time.time() - t1
    del e, w
    roots = O.generate_bfs_roots(rs, n, 2, 3, 64).tolist()
    K, W = args.steps, args.warmup
    seq = [roots[i % len(roots)] for i in range(W + K)]
    nedge = {}
    pred = np.empty(n, np.int64)
    depth = np.empty(n, np.int64)
    for r in seq[:W]:
        O.bfs_clear(n, pred, depth)
        O.bfs_search(rs, col, n, r, pred, depth)
        nedge[r] = O.edge_count(rs, col, n, pred)
    secs = []
    t_start = time.perf_counter()
    for r in seq[W:]:
        O.bfs_clear(n, pred, depth)  # untimed, as the runner's oned_graph_bfs_clear
        t = time.perf_counter()
        O.bfs_search(rs, col, n, r, pred, depth)
        secs.append(time.perf_counter() - t)
        if r not in nedge:
            nedge[r] = O.edge_count(rs, col, n, pred)
    total = time.perf_counter() - t_start
    timed = seq[W:]
    v = hmean_gteps([nedge[r] for r in timed], secs)
    line = {
        "metric": metric_name(scale, ef), "value": float(f"{v:.6g}"), "unit": "GTEPS", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": round(total / K * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic: Graph500 Kronecker generator, seeds (2,3)",
        "config": bench_config(scale, ef, K, world, int(rs[-1])),
        "impl": "reference",
        "median_gteps": round(float(np.median(np.asarray([nedge[r] for r in timed]) / np.asarray(secs) / 1e9)), 4),
        "cpu_baseline": {"value": float(f"{v:.6g}"), "unit": "GTEPS", "cores": O.num_threads(), "kind": "port",
                         "sample": f"{K} BFS roots; the reference has no CPU path, so this is its top-down "
                                   "algorithm as restated in oracle/ (OpenMP)"},
        "e2e": {"value": float(f"{v:.6g}"), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "setup": {"generation_s": round(gen_s, 1), "csr_build_s": round(csr_s, 1)},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--scale", type=int, default=26)
    ap.add_argument("--edgefactor", type=int, default=16)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-roots", type=int, default=0,
                    help="timed roots the CPU baseline searches (and compares depth arrays for); 0 = all")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU build (oracle/_ref/ref_bench) on the same roots")
    ap.add_argument("--batched-scale", type=int, default=24, help="SCALE of the batched (multi-source) BFS graph")
    ap.add_argument("--sssp-batched-scale", type=int, default=18,
                    help="SCALE of the batched SSSP graph (32 sources in one launch)")
    ap.add_argument("--batched-roots", type=int, default=256)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched BFS measurement")
    ap.add_argument("--only-batched", nargs="?", const="msbfs", choices=["msbfs", "sssp", "packed", "serve", "all"],
                    help="run only the batched measurements (multi-source BFS, packed graphs, serving or all)")
    ap.add_argument("--serve-queries", type=int, default=2000)
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="Poisson arrival rate, queries per second")
    ap.add_argument("--serve-slots", type=int, default=8, help="concurrent launches (streams) of the server")
    ap.add_argument("--serve-count-errors", action="store_true",
                    help="serving: count launches that report a device error instead of raising")
    ap.add_argument("--serve-low-rate", type=float, default=250.0,
                    help="rate of the second, below-capacity serving trace (0 = skip it)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving measurement")
    ap.add_argument("--packed-graphs", type=int, default=2000)
    ap.add_argument("--packed-min-scale", type=int, default=10)
    ap.add_argument("--packed-max-scale", type=int, default=18)
    ap.add_argument("--no-packed", action="store_true", help="skip the packed many-graph measurement")
    ap.add_argument("--no-tune", action="store_true", help="headline searches on the library's default knobs")
    ap.add_argument("--tune-cache", default=os.path.join(REPO, "cuda-graph-traversal_b200", "tuned.json"),
                    help="JSON cache of the headline searches' tuned knobs (keyed by device and graph size)")
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu dram bytes per BFS launch (read+write) to report beside the roofline")
    ap.add_argument("--kernels-once", type=int, default=0, metavar="SCALE",
                    help="one pass of every kernel of the path at SCALE (the command the ncu summaries profile): "
                         "generation, canonical CSR, SSSP and BFS copies, one BFS and SSSP from a main-component "
                         "root, the edge count and both validations")
    args = ap.parse_args()
    if args.warmup < 1 or args.steps < 1:
        ap.error("steps and warmup must be positive")
    if args.impl == "reference":
        run_reference(args)
    elif args.kernels_once:
        run_kernels_once(args.kernels_once, args.edgefactor)
    elif args.only_batched:
        run_batched_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
