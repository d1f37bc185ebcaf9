"""numpy/ctypes front end of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA library and the
timed CPU baseline of ``bench.py``.  Only ``tests/``, ``__graft_entry__.smoke``
and ``bench.py`` (its CPU-baseline and ``--impl reference`` legs) import this
module; the product never does.  Each function names the reference code it
restates (see ``g500_oracle.c`` for the line-level citations).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile liboracle.so with oracle/Makefile (gcc + OpenMP)."""
    src = os.path.join(_HERE, "g500_oracle.c")
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    L = C.CDLL(build())
    L.orc_make_mrg_seed.argtypes = [C.c_uint64, C.c_uint64, u32p]
    L.orc_make_random_numbers.argtypes = [C.c_int64, C.c_uint64, C.c_uint64, C.c_int64, f64p]
    L.orc_scramble_keys.argtypes = [u32p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.orc_generate_kronecker_range.argtypes = [u32p, C.c_int, C.c_int64, C.c_int64, u64p, f32p, C.c_int]
    L.orc_csr_count.argtypes = [u64p, C.c_uint64, C.c_uint64, u64p, C.c_int]
    L.orc_csr_count.restype = C.c_uint64
    L.orc_csr_build.argtypes = [u64p, f32p, C.c_uint64, C.c_uint64, u64p, u32p, f32p, C.c_int, C.c_int]
    L.orc_generate_bfs_roots.argtypes = [u64p, C.c_uint64, C.c_uint64, C.c_uint64, u64p, C.c_int]
    L.orc_generate_bfs_roots.restype = C.c_int
    L.orc_bfs.argtypes = [u64p, u32p, C.c_uint64, C.c_uint64, i64p, i64p, C.c_int]
    L.orc_bfs.restype = C.c_int
    L.orc_bfs_clear.argtypes = [C.c_uint64, i64p, i64p, C.c_int]
    L.orc_bfs_search.argtypes = [u64p, u32p, C.c_uint64, C.c_uint64, i64p, i64p, C.c_int]
    L.orc_bfs_search.restype = C.c_int
    L.orc_bfs_dist_from_pred.argtypes = [u64p, u32p, C.c_uint64, i64p, C.c_uint64, i64p]
    L.orc_bfs_validate.argtypes = [u64p, u32p, C.c_uint64, C.c_uint64, i64p, i64p]
    L.orc_bfs_validate.restype = C.c_uint64
    L.orc_edge_count.argtypes = [u64p, u32p, C.c_uint64, i64p]
    L.orc_edge_count.restype = C.c_uint64
    L.orc_sssp.argtypes = [u64p, u32p, f32p, C.c_uint64, C.c_uint64, f32p, i64p]
    L.orc_sssp_validate.argtypes = [u64p, u32p, f32p, C.c_uint64, C.c_uint64, f32p, i64p]
    L.orc_sssp_validate.restype = C.c_uint64
    L.orc_num_threads.restype = C.c_int
    _lib = L
    return L


def num_threads() -> int:
    return lib().orc_num_threads()


def make_mrg_seed(s1: int, s2: int) -> np.ndarray:
    """make_mrg_seed (src/graph_generation.cu:248-254)."""
    out = np.zeros(5, np.uint32)
    lib().orc_make_mrg_seed(s1, s2, out)
    return out


def make_random_numbers(n: int, s1: int, s2: int, position: int) -> np.ndarray:
    """make_random_numbers (src/graph_generation.cu:256-266)."""
    out = np.zeros(n, np.float64)
    lib().orc_make_random_numbers(n, s1, s2, position, out)
    return out


def scramble_keys(seed: np.ndarray) -> tuple[int, int]:
    """The two scrambling keys (src/graph_generation.cu:290-300)."""
    a, b = C.c_uint64(), C.c_uint64()
    lib().orc_scramble_keys(np.ascontiguousarray(seed, np.uint32), C.byref(a), C.byref(b))
    return a.value, b.value


def generate_kronecker_range(seed: np.ndarray, scale: int, start: int, end: int,
                             nthreads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Edges [start, end) as an (n, 2) uint64 array plus float32 weights
    (generate_kronecker_range, src/graph_generation.cu:269-310)."""
    n = max(end - start, 0)
    edges = np.zeros((n, 2), np.uint64)
    w = np.zeros(n, np.float32)
    if n:
        lib().orc_generate_kronecker_range(np.ascontiguousarray(seed, np.uint32), scale, start, end,
                                           edges.reshape(-1), w, nthreads)
    return edges, w


def csr_build(edges: np.ndarray, w: np.ndarray, nverts: int, canonical: bool = True,
              nthreads: int = 0) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """CSR (rowstarts u64[N+1], col u32[E], w f32[E]) of
    oned_graph_from_tuple_graph (src/traversal.cu:342-389); rows sorted by
    (dst, weight bits) when ``canonical``."""
    e = np.ascontiguousarray(edges, np.uint64).reshape(-1)
    m = e.size // 2
    deg = np.zeros(nverts, np.uint64)
    total = lib().orc_csr_count(e, m, nverts, deg, nthreads)
    rowstarts = np.zeros(nverts + 1, np.uint64)
    col = np.zeros(max(total, 1), np.uint32)
    wo = np.zeros(max(total, 1), np.float32)
    lib().orc_csr_build(e, np.ascontiguousarray(w, np.float32), m, nverts, rowstarts, col, wo,
                        1 if canonical else 0, nthreads)
    return rowstarts, col[:total], wo[:total]


def generate_bfs_roots(rowstarts: np.ndarray, nverts: int, s1: int = 2, s2: int = 3,
                       max_roots: int = 64) -> np.ndarray:
    """generate_bfs_roots (examples/graph500_runner.cu:43-74)."""
    out = np.zeros(max_roots, np.uint64)
    n = lib().orc_generate_bfs_roots(rowstarts, nverts, s1, s2, out, max_roots)
    return out[:n]


def _col(col):
    return np.ascontiguousarray(col, np.uint32)


def bfs(rowstarts, col, nverts: int, root: int, nthreads: int = 0):
    """Top-down BFS (bfs_run_kernel, src/traversal.cu:139-207) -> (pred, depth)."""
    pred = np.zeros(nverts, np.int64)
    depth = np.zeros(nverts, np.int64)
    lib().orc_bfs(rowstarts, _col(col), nverts, root, pred, depth, nthreads)
    return pred, depth


def bfs_clear(nverts: int, pred: np.ndarray, depth: np.ndarray, nthreads: int = 0) -> None:
    """The clear half of bfs (the runner's untimed oned_graph_bfs_clear)."""
    lib().orc_bfs_clear(nverts, pred, depth, nthreads)


def bfs_search(rowstarts, col, nverts: int, root: int, pred: np.ndarray, depth: np.ndarray,
               nthreads: int = 0) -> int:
    """The search half of bfs on cleared arrays; returns the level count."""
    return lib().orc_bfs_search(rowstarts, _col(col), nverts, root, pred, depth, nthreads)


def bfs_dist_from_pred(rowstarts, col, nverts: int, pred: np.ndarray, root: int) -> np.ndarray:
    """bfs_compute_dist_from_pred (src/traversal.cu:505-563)."""
    dist = np.zeros(nverts, np.int64)
    lib().orc_bfs_dist_from_pred(rowstarts, _col(col), nverts, np.ascontiguousarray(pred, np.int64),
                                 root, dist)
    return dist


def bfs_validate(rowstarts, col, nverts: int, root: int, pred, dist) -> int:
    """Error count of the runner's 7 BFS rules (examples/graph500_runner.cu:84-169)."""
    return lib().orc_bfs_validate(rowstarts, _col(col), nverts, root,
                                  np.ascontiguousarray(pred, np.int64),
                                  np.ascontiguousarray(dist, np.int64))


def edge_count(rowstarts, col, nverts: int, pred) -> int:
    """TEPS edge count (examples/graph500_runner.cu:171-201)."""
    return lib().orc_edge_count(rowstarts, _col(col), nverts, np.ascontiguousarray(pred, np.int64))


def sssp(rowstarts, col, w, nverts: int, root: int):
    """float32 shortest paths (oned_graph_sssp_run semantics,
    src/traversal.cu:638-711) -> (dist f32 with -1 unreached, pred i64)."""
    dist = np.zeros(nverts, np.float32)
    pred = np.zeros(nverts, np.int64)
    lib().orc_sssp(rowstarts, _col(col), np.ascontiguousarray(w, np.float32), nverts, root, dist, pred)
    return dist, pred


def sssp_validate(rowstarts, col, w, nverts: int, root: int, dist, pred) -> int:
    """Error count of the SSSP rules in g500_oracle.c (the reference has none)."""
    return lib().orc_sssp_validate(rowstarts, _col(col), np.ascontiguousarray(w, np.float32),
                                   nverts, root, np.ascontiguousarray(dist, np.float32),
                                   np.ascontiguousarray(pred, np.int64))
