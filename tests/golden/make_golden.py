"""Generates the golden fixtures in this directory from the reference itself.

Two sources, both built from the reference's own sources by oracle/ref.mk:

  host   oracle/_ref/libref_host.so -- the reference's src/graph_generation.cu
         compiled for the host (its MRG jump over the generated table of
         src/mrg_transitions.cu, its step, make_mrg_seed and
         make_random_numbers).  Runs here:
             python tests/golden/make_golden.py host

  dumps  oracle/_ref/ref_dump -- the reference library (generator, CSR,
         BFS + bfs_compute_dist_from_pred, delta-stepping SSSP) run on one
         GPU with the single-process MPI/NVSHMEM shims of include/compat/shim.
         Run on a GPU machine, e.g.
             oracle/_ref/ref_dump 12 16 64 OUT12 && oracle/_ref/ref_dump 14 16 16 OUT14
         then here:
             python tests/golden/make_golden.py dumps 12 OUT12 14 OUT14

Outputs: ref_host_kat.json, ref_s<SCALE>.json (+ ref_s12_depth.npz).  The
hashes are defined in golden_hashes() below and recomputed by the tests.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def canonical_csr(rowstarts, col, w):
    """Rows sorted by (dst, weight bits): the reference's in-row order
    depends on atomic order, so CSRs are compared in this form."""
    rs = np.asarray(rowstarts).astype(np.int64)
    n = rs.size - 1
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(rs))
    wb = np.asarray(w, np.float32).view(np.uint32)
    c = np.asarray(col).astype(np.int64)
    order = np.lexsort((wb, c, src))
    return c[order].astype(np.uint32), wb[order]


def golden_hashes(edges, weights, rowstarts, col, w):
    cc, cw = canonical_csr(rowstarts, col, w)
    return {
        "edges_sha256": sha(np.asarray(edges, np.uint64)),
        "weights_sha256": sha(np.asarray(weights, np.float32)),
        "rowstarts_sha256": sha(np.asarray(rowstarts, np.uint64)),
        "csr_canonical_sha256": sha(cc, cw),
    }


def host_kats() -> dict:
    lib = C.CDLL(os.path.join(REPO, "oracle", "_ref", "libref_host.so"))
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    lib.ref_mrg_skip.argtypes = [u32p, C.c_uint64, C.c_uint64, C.c_uint64]
    lib.ref_mrg_draw.argtypes = [u32p, C.c_int, u32p]
    lib.ref_make_mrg_seed.argtypes = [C.c_uint64, C.c_uint64, u32p]
    lib.ref_make_random_numbers.argtypes = [C.c_int64, C.c_uint64, C.c_uint64, C.c_int64, f64p]
    rng = np.random.default_rng(20260101)
    out = {"source": "oracle/_ref/libref_host.so (reference src/graph_generation.cu, host side)"}
    seeds = []
    for s1, s2 in [(2, 3), (0, 0), (1, 1), (12345, 67890), (2**63 + 5, 2**62 + 7), (2**64 - 1, 2**64 - 1)]:
        o = np.zeros(5, np.uint32)
        lib.ref_make_mrg_seed(s1, s2, o)
        seeds.append({"s1": s1, "s2": s2, "seed": o.tolist()})
    out["make_mrg_seed"] = seeds
    rn = []
    for s1, s2, pos in [(2, 3, 0), (2, 3, 1), (2, 3, 2), (2, 3, 1000), (2, 3, 2**20 + 3), (7, 11, 123456789)]:
        o = np.zeros(8, np.float64)
        lib.ref_make_random_numbers(8, s1, s2, pos, o)
        rn.append({"s1": s1, "s2": s2, "position": pos, "values_hex": [float(x).hex() for x in o]})
    out["make_random_numbers"] = rn
    skips = []
    for i in range(96):
        z = rng.integers(1, 2**31 - 1, 5).astype(np.uint32)
        hi, mid, lo = [int(x) for x in rng.integers(0, 2**63, 3, dtype=np.uint64)]
        if i % 4 == 0:
            hi = 0
        if i % 4 == 1:
            hi, lo = 0, 0
        r = z.copy()
        lib.ref_mrg_skip(r, hi, mid, lo)
        skips.append({"state": z.tolist(), "high": hi, "mid": mid, "low": lo, "result": r.tolist()})
    out["mrg_skip"] = skips
    # Scrambling keys as generate_kronecker_range derives them
    # (src/graph_generation.cu:290-300): jump 50*2^128 + 7*2^64, four draws.
    keys = []
    for s1, s2 in [(2, 3), (12345, 67890)]:
        seed = np.zeros(5, np.uint32)
        lib.ref_make_mrg_seed(s1, s2, seed)
        z = seed.copy()
        lib.ref_mrg_skip(z, 50, 7, 0)
        d = np.zeros(4, np.uint32)
        lib.ref_mrg_draw(z, 4, d)
        v0 = (int(d[0]) * 0xFFFFFFFF + int(d[1])) % 2**64
        v1 = (int(d[2]) * 0xFFFFFFFF + int(d[3])) % 2**64
        keys.append({"s1": s1, "s2": s2, "val0": v0, "val1": v1})
    out["scramble_keys"] = keys
    draws = np.zeros(64, np.uint32)
    z = np.array([3, 1, 4, 1, 1], np.uint32)
    lib.ref_mrg_draw(z, 64, draws)
    out["mrg_draws_from_seed_2_3"] = draws.tolist()
    return out


def dump_fixture(scale: int, d: str) -> tuple[dict, np.ndarray]:
    n = 1 << scale

    def rd(name, t):
        return np.fromfile(os.path.join(d, name), t)

    edges = rd("edges.u64", np.uint64).reshape(-1, 2)
    weights = rd("weights.f32", np.float32)
    rowstarts = rd("rowstarts.u64", np.uint64)
    column = rd("column.u64", np.uint64)
    csrw = rd("csrw.f32", np.float32)
    roots = rd("roots.u64", np.uint64)
    pred = rd("bfs_pred.i64", np.int64).reshape(-1, n)
    dist = rd("bfs_dist.i64", np.int64).reshape(-1, n)
    sdist = rd("sssp_dist.f32", np.float32).reshape(-1, n)
    fx = {
        "source": "oracle/_ref/ref_dump (reference sources + single-process shims) on one B200",
        "scale": scale,
        "edgefactor": edges.shape[0] >> scale,
        "seeds": [2, 3],
        "nedges": int(edges.shape[0]),
        "nentries": int(rowstarts[-1]),
        "first_edges": edges[:16].tolist(),
        "first_weights_hex": [float(x).hex() for x in weights[:16]],
        "self_loops": int((edges[:, 0] == edges[:, 1]).sum()),
        "isolated": int((np.diff(rowstarts.astype(np.int64)) == 0).sum()),
        "max_degree": int(np.diff(rowstarts.astype(np.int64)).max()),
        "roots": roots.tolist(),
    }
    fx.update(golden_hashes(edges, weights, rowstarts, column, csrw))
    per = []
    for i, r in enumerate(roots.tolist()):
        src = np.repeat(np.arange(n, dtype=np.int64), np.diff(rowstarts.astype(np.int64)))
        reached_rows = pred[i][src] != -1
        nedge = int(np.count_nonzero(reached_rows & (column.astype(np.int64) <= src)))
        per.append({
            "root": r,
            "nedge": nedge,
            "reached": int(np.count_nonzero(pred[i] != -1)),
            "max_depth": int(dist[i].max()),
            "depth_sha256": sha(dist[i]),
            "sssp_dist_sha256": sha(sdist[i]),
            "sssp_reached": int(np.count_nonzero(sdist[i] != -1.0)),
            "sssp_dist_max_hex": float(sdist[i].max()).hex(),
        })
    fx["per_root"] = per
    return fx, dist.astype(np.int8)


def main(argv):
    if not argv or argv[0] not in ("host", "dumps"):
        print(__doc__)
        return 2
    if argv[0] == "host":
        with open(os.path.join(HERE, "ref_host_kat.json"), "w") as f:
            json.dump(host_kats(), f, indent=1)
        return 0
    pairs = argv[1:]
    for scale, d in zip(pairs[0::2], pairs[1::2]):
        fx, depth = dump_fixture(int(scale), d)
        with open(os.path.join(HERE, f"ref_s{scale}.json"), "w") as f:
            json.dump(fx, f, indent=1)
        if int(scale) == 12:
            np.savez_compressed(os.path.join(HERE, "ref_s12_depth.npz"), depth=depth)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
