"""Python host mirror of the reference's Graph500 API over libg500b.so.

The functions keep the names, argument meaning and error behaviour of the
reference's C++ API (src/graph_generation.h, src/traversal.h and the
runner's helpers in examples/graph500_runner.cu); the work runs in the CUDA
kernels of libg500b.so through its C ABI (include/g500b.h).  PyTorch only
provides device memory and the current stream.  There is no CPU path: if the
shared library is missing, importing this module raises.

Layout on the device (one graph):
  rowstarts  uint64[N+1]   stored as torch.int64
  col        int32[E]      neighbour ids, light entries (w < delta) first in each row
  w          float32[E]
  light_deg  int32[N]      light entries per row (uint32 on the C side)
  column     int64[E]      optional u64 copy of col (the reference's Oned_Graph.column)
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libg500b.so")

G5_OK = 0
class G5Error(RuntimeError):
    """Any error the library returned (also raised as the matching builtin
    kind below)."""


class G5InvalidError(G5Error, ValueError):
    pass


class G5WorkspaceError(G5Error, MemoryError):
    pass


class G5CudaError(G5Error):
    pass


class G5TimeoutError(G5Error, TimeoutError):
    pass


class G5DeviceError(G5Error):
    pass


_ERRORS = {-1: G5InvalidError, -2: G5WorkspaceError, -3: G5CudaError, -4: G5TimeoutError, -5: G5DeviceError}


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libg500b.so not built at {LIB_PATH}; run `make -C {_HERE}` "
                          "(or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    p, u64, i64, u32, i32, f32 = C.c_void_p, C.c_uint64, C.c_int64, C.c_uint32, C.c_int32, C.c_float
    sig = {
        "g5_last_error": ([], C.c_char_p),
        "g5_version": ([], C.c_char_p),
        "g5_make_mrg_seed": ([u64, u64, p], C.c_int),
        "g5_make_random_numbers": ([i64, u64, u64, i64, p], C.c_int),
        "g5_scramble_keys": ([p, p, p], C.c_int),
        "g5_generate_kronecker_range": ([p, u32, i64, i64, p, p, p], C.c_int),
        "g5_csr_workspace_size": ([u64, u64, p], C.c_int),
        "g5_csr_count": ([p, u64, u64, p, p, u64, p, p], C.c_int),
        "g5_csr_fill": ([p, p, u64, u64, p, f32, p, u64, p, p, p, p, p], C.c_int),
        "g5_csr_count_kronecker": ([p, u32, u64, p, p, u64, p, p], C.c_int),
        "g5_csr_fill_kronecker": ([p, u32, u64, p, f32, p, u64, p, p, p, p, p], C.c_int),
        "g5_csr_pack_append": ([p, p, p, p, u64, u64, u64, u64, p, p, p, p, p], C.c_int),
        "g5_csr_split_tiny": ([p, p, p, p, p, u64, f32, p, p], C.c_int),
        "g5_csr_sorted_workspace_size": ([u64, u64, p], C.c_int),
        "g5_csr_fill_sorted": ([p, p, u64, u64, p, u64, p, u64, p, p, p, p], C.c_int),
        "g5_csr_radix_workspace_size": ([u64, u64, p], C.c_int),
        "g5_csr_radix_count": ([p, u64, u64, p, u64, p, p], C.c_int),
        "g5_csr_radix_fill": ([p, p, u64, u64, u64, p, u64, p, p, p, p, p], C.c_int),
        "g5_csr_sort_rows": ([p, u64, u64, p, p, p, p, u64, p], C.c_int),
        "g5_csr_degree_order_workspace_size": ([u64, u64, p], C.c_int),
        "g5_csr_degree_order": ([p, p, u64, u64, p, p, u64, p], C.c_int),
        "g5_csr_sssp_renumber_workspace_size": ([u64, p], C.c_int),
        "g5_csr_sssp_renumber": ([p, p, p, p, p, u64, u64, p, p, p, p, p, p, p, p, u64, p], C.c_int),
        "g5_csr_dedupe_count": ([p, p, u64, u64, p, p, u64, p, p], C.c_int),
        "g5_csr_dedupe_copy": ([p, p, p, u64, p, p, p, p, p], C.c_int),
        "g5_csr_split_light": ([p, p, p, u64, u64, f32, p, p, p, p, p, u64, p], C.c_int),
        "g5_bfs_traverse_multi": ([p, p, u64, p, u32, p, p, p, u64, p, p], C.c_int),
        "g5_sssp_traverse_multi": ([p, p, p, p, f32, u64, p, u32, p, p, p, u64, p, p], C.c_int),
        "g5_bfs_workspace_size": ([u64, p], C.c_int),
        "g5_bfs_run": ([p, p, u64, u64, p, p, p, u64, p, p], C.c_int),
        "g5_bfs_reset": ([u64, p, p, p, p, u64, p], C.c_int),
        "g5_bfs_reset_touched": ([u64, p, p, p, p, u64, p], C.c_int),
        "g5_graph_isolated_bitmap": ([p, u64, p, p], C.c_int),
        "g5_bfs_traverse": ([p, p, u64, u64, p, p, p, u64, p, p], C.c_int),
        "g5_bfs_query": ([p, p, u64, p, p, p, p, p, u64, p, p, p], C.c_int),
        "g5_bfs_export": ([p, p, u64, p, u64, p, u64, p, p], C.c_int),
        "g5_bfs_first_neighbours": ([p, p, u64, p, p], C.c_int),
        "g5_bfs_query_plan_create": ([p, p, u64, p, p, p, p, u64, p, p, p, p], C.c_int),
        "g5_bfs_query_plan_run": ([p, u64], C.c_int),
        "g5_bfs_query_plan_export": ([p, u64, p, u64, p], C.c_int),
        "g5_bfs_query_plan_destroy": ([p], None),
        "g5_bfs_visited_bitmap": ([p, u64, u64, p, p], C.c_int),
        "g5_bfs_last_stats": ([p, u64, p, p], C.c_int),
        "g5_bfs_last_trace": ([p, u64, C.c_int, p, p, p, p, p, p, p], C.c_int),
        "g5_bfs_dist_from_pred": ([p, p, u64, p, u64, p, p, u64, p], C.c_int),
        "g5_sssp_workspace_size": ([u64, p], C.c_int),
        "g5_sssp_run": ([p, p, p, p, f32, u64, u64, p, p, p, u64, p, p], C.c_int),
        "g5_sssp_multi_workspace_size": ([u64, p], C.c_int),
        "g5_sssp_multi_last_stats": ([p, u64, p, p], C.c_int),
        "g5_sssp_multi_grid": ([u64, p, p], C.c_int),
        "g5_sssp_multi_run": ([p, p, p, u64, p, p, p, C.c_uint32, p, p, p, u64, C.c_float, C.c_int32, p, p],
                              C.c_int),
        "g5_sssp_last_status": ([p, u64, p, p, p], C.c_int),
        "g5_sssp_reset": ([u64, p, p, p, u64, p], C.c_int),
        "g5_sssp_reset_touched": ([u64, p, p, p, u64, p], C.c_int),
        "g5_sssp_last_trace": ([p, u64, p, C.c_int, p, p, p, p, p, p], C.c_int),
        "g5_sssp_traverse": ([p, p, p, p, f32, u64, u64, p, p, p, u64, p, p], C.c_int),
        "g5_validate_workspace_size": ([u64, p], C.c_int),
        "g5_edge_count": ([p, p, u64, p, p, u64, p, p], C.c_int),
        "g5_bfs_validate": ([p, p, u64, u64, p, p, p, u64, p, p], C.c_int),
        "g5_sssp_validate": ([p, p, p, u64, u64, p, p, p, u64, p, p], C.c_int),
        "g5_bfs_validate_renumbered": ([p, p, u64, u64, p, p, p, p, p, u64, p, p], C.c_int),
        "g5_sssp_validate_renumbered": ([p, p, p, u64, u64, p, p, p, p, p, u64, p, p], C.c_int),
        "g5_selftest_wait_timeout": ([u32, p, u64, p], C.c_int),
        "g5_msbfs_workspace_size": ([u64, u64, C.c_int, p], C.c_int),
        "g5_bfs_grid": ([u64, p, p], C.c_int),
        "g5_sssp_grid": ([u64, p, p], C.c_int),
        "g5_msbfs_grid": ([u64, p, p], C.c_int),
        "g5_msbfs_prepare": ([p, p, u64, u64, C.c_int, p, u64, p], C.c_int),
        "g5_msbfs_run": ([u64, u64, C.c_int, p, u32, p, u64, p, p, p], C.c_int),
        "g5_msbfs_depths_u8": ([p, u64, u64, u64, C.c_int, u32, p, p], C.c_int),
        "g5_msbfs_depth": ([p, u64, u64, u64, C.c_int, u32, p, p], C.c_int),
        "g5_msbfs_last_stats": ([p, u64, p, p], C.c_int),
        "g5_msbfs_last_trace": ([p, u64, C.c_int, p, p, p, p, p, p], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


lib = _load()
_plan_run = lib.g5_bfs_query_plan_run
_plan_export = lib.g5_bfs_query_plan_export


def _check(rc: int) -> None:
    if rc != G5_OK:
        msg = lib.g5_last_error().decode()
        raise _ERRORS.get(rc, G5Error)(f"libg500b error {rc}: {msg}")


class BfsParams(C.Structure):
    _fields_ = [("alpha", C.c_float), ("beta", C.c_float), ("mode", C.c_int32), ("blocks", C.c_int32),
                ("big_deg", C.c_int32), ("chunk", C.c_int32), ("lane_entries", C.c_int32), ("top", C.c_void_p)]


class BfsStats(C.Structure):
    _fields_ = [("levels", C.c_int32), ("bottom_up_levels", C.c_int32), ("reached", C.c_uint64),
                ("error_flags", C.c_uint32), ("solo_levels", C.c_int32)]


class MsBfsParams(C.Structure):
    _fields_ = [("alpha", C.c_float), ("mode", C.c_int32), ("check_frontier", C.c_int32), ("blocks", C.c_int32)]


class MsBfsStats(C.Structure):
    _fields_ = [("levels", C.c_int32), ("pull_levels", C.c_int32), ("error_flags", C.c_uint32),
                ("nroots", C.c_uint32), ("pairs_reached", C.c_uint64), ("frontier_edges", C.c_uint64)]


class SsspMultiStats(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("error_flags", C.c_uint32), ("frontier_entries", C.c_uint64),
                ("entries_scanned", C.c_uint64)]


class SsspParams(C.Structure):
    _fields_ = [("delta", C.c_float), ("blocks", C.c_int32), ("pull", C.c_float), ("sub_min", C.c_int32),
                ("small", C.c_int32), ("tiny_deg", C.c_void_p), ("check_opens", C.c_int32), ("big_deg", C.c_int32),
                ("chunk", C.c_int32), ("perm", C.c_void_p), ("inv", C.c_void_p)]


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)
_cur_dev = getattr(torch._C, "_cuda_getDevice", None)


def _stream(stream=None) -> int | None:
    if stream is not None:
        return stream.cuda_stream or None
    if _raw_stream is not None and _cur_dev is not None:
        return _raw_stream(_cur_dev()) or None  # the current stream without building a Stream object
    return torch.cuda.current_stream().cuda_stream or None


def _workspace(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def search_grid(kind: str, nverts: int) -> tuple[int, int]:
    """(blocks, max co-resident blocks) of the persistent kernel of `kind`
    ("bfs", "sssp", "msbfs", "sssp_multi") for a graph of nverts vertices."""
    b, m = C.c_int32(), C.c_int32()
    _check(getattr(lib, f"g5_{kind}_grid")(nverts, C.byref(b), C.byref(m)))
    return b.value, m.value


def version() -> str:
    return lib.g5_version().decode()


def selftest_wait_timeout(limit_ms: int = 50, device="cuda") -> None:
    """Runs the bounded-wait self test; raises TimeoutError as designed."""
    work = torch.zeros(64, dtype=torch.uint8, device=device)
    _check(lib.g5_selftest_wait_timeout(limit_ms, _ptr(work), work.numel(), _stream()))


# ----------------------------------------------------------------- MRG ----

def make_mrg_seed(userseed1: int, userseed2: int) -> list[int]:
    """make_mrg_seed (src/graph_generation.h:39)."""
    seed = (C.c_uint32 * 5)()
    _check(lib.g5_make_mrg_seed(userseed1, userseed2, seed))
    return list(seed)


def make_random_numbers(nvalues: int, userseed1: int, userseed2: int, position: int) -> np.ndarray:
    """make_random_numbers (src/graph_generation.h:40)."""
    out = np.zeros(max(nvalues, 0), np.float64)
    _check(lib.g5_make_random_numbers(nvalues, userseed1, userseed2, position,
                                      out.ctypes.data if nvalues else None))
    return out


def scramble_keys(seed) -> tuple[int, int]:
    s = (C.c_uint32 * 5)(*seed)
    a, b = C.c_uint64(), C.c_uint64()
    _check(lib.g5_scramble_keys(s, C.byref(a), C.byref(b)))
    return a.value, b.value


# ----------------------------------------------------------- generator ----

@dataclass
class TupleGraph:
    """Tuple_Graph (src/graph_generation.h:12-19): edges (M, 2) as int64
    holding the u64 vertex ids, weights float32[M]."""
    edges: torch.Tensor
    weights: torch.Tensor
    nglobaledges: int

    @property
    def edges_size(self) -> int:
        return self.edges.shape[0]


def generate_kronecker_range(seed, log_n: int, start_edge: int, end_edge: int,
                             device="cuda", out: TupleGraph | None = None, stream=None) -> TupleGraph:
    """generate_kronecker_range (src/graph_generation.h:33-37)."""
    m = max(end_edge - start_edge, 0)
    if out is None:
        out = TupleGraph(torch.empty((m, 2), dtype=torch.int64, device=device),
                         torch.empty(m, dtype=torch.float32, device=device), m)
    s = (C.c_uint32 * 5)(*seed)
    _check(lib.g5_generate_kronecker_range(s, log_n, start_edge, end_edge, _ptr(out.edges),
                                           _ptr(out.weights), _stream(stream)))
    return out


# ----------------------------------------------------------------- CSR ----

@dataclass
class OnedGraph:
    """Oned_Graph (src/traversal.h:8-16) at one rank, plus the int32 column
    and per-row light counts the kernels use."""
    nglobalverts: int
    nlocaledges: int
    rowstarts: torch.Tensor
    col: torch.Tensor
    w: torch.Tensor
    light_deg: torch.Tensor
    light_delta: float
    column: torch.Tensor | None = None
    isolated: torch.Tensor | None = None  # int32[ceil(N/32)] bitmap of degree-0 vertices
    main_bits: np.ndarray | None = None   # host uint32 bitmap of the largest component
    tiny_deg: torch.Tensor | None = None  # int32[N] leading tiny entries of each light part
    # The SSSP copy (g5_csr_split_light): rows partitioned tiny | light |
    # heavy, light_deg / tiny_deg their first parts' sizes.  None: col / w
    # are in that layout themselves (packed graphs).
    scol: torch.Tensor | None = None
    sw: torch.Tensor | None = None
    # The BFS copy of the column (g5_csr_degree_order): each row's
    # neighbours by decreasing degree.  None: the BFS reads col.
    bcol: torch.Tensor | None = None
    # Each vertex's first entry of bcol (g5_bfs_first_neighbours): what a
    # bottom-up level probes before reading the row.
    btop: torch.Tensor | None = None
    # The SSSP copy renumbered by decreasing degree (g5_csr_sssp_renumber),
    # which the SSSP entry points use when present; None: the split copy
    # above in the caller's numbering.
    sr: "SsspCopy | None" = None

    @property
    def bfs_col(self) -> torch.Tensor:
        return self.col if self.bcol is None else self.bcol

    @property
    def sssp_col(self) -> torch.Tensor:
        return self.col if self.scol is None else self.scol

    @property
    def sssp_w(self) -> torch.Tensor:
        return self.w if self.sw is None else self.sw

    def in_main_component(self, v: int) -> bool:
        """True when v is in the largest component (or unknown / out of
        range: the library call itself then validates v)."""
        if self.main_bits is None or not 0 <= v < self.nglobalverts:
            return True
        return bool((int(self.main_bits[v >> 5]) >> (v & 31)) & 1)

    @property
    def nlocalverts(self) -> int:
        return self.nglobalverts

    @property
    def device(self):
        return self.rowstarts.device


@dataclass
class SsspCopy:
    """The SSSP's CSR in its own vertex numbering (decreasing degree): row
    starts, column, weights, light and tiny counts, perm (caller's vertex ->
    search's) and inv (back)."""
    rowstarts: torch.Tensor
    col: torch.Tensor
    w: torch.Tensor
    light_deg: torch.Tensor
    tiny_deg: torch.Tensor
    perm: torch.Tensor
    inv: torch.Tensor


def oned_graph_sssp_renumber(g: OnedGraph, stream=None) -> OnedGraph:
    """Gives the SSSP a copy of its split CSR renumbered by decreasing
    degree (g5_csr_sssp_renumber): the vertices most relaxations target
    then have their per-vertex state side by side, where it stays in L2.
    Distances are unchanged; parents are still tight edges' sources.  Costs
    12 bytes per CSR entry and 24 per vertex."""
    n, e = g.nglobalverts, g.nlocaledges
    dev = g.device
    nb = C.c_uint64()
    _check(lib.g5_csr_sssp_renumber_workspace_size(n, C.byref(nb)))
    work = _workspace(nb.value, dev)
    i32 = dict(dtype=torch.int32, device=dev)
    sr = SsspCopy(torch.empty(n + 1, dtype=torch.int64, device=dev), torch.empty(max(e, 1), **i32),
                  torch.empty(max(e, 1), dtype=torch.float32, device=dev), torch.empty(n, **i32), torch.empty(n, **i32),
                  torch.empty(n, **i32), torch.empty(n, **i32))
    _check(lib.g5_csr_sssp_renumber(_ptr(g.rowstarts), _ptr(g.sssp_col), _ptr(g.sssp_w), _ptr(g.light_deg),
                                    _ptr(g.tiny_deg), n, e, _ptr(sr.perm), _ptr(sr.inv), _ptr(sr.rowstarts),
                                    _ptr(sr.col), _ptr(sr.w), _ptr(sr.light_deg), _ptr(sr.tiny_deg), _ptr(work),
                                    work.numel(), _stream(stream)))
    g.sr = sr
    return g


def _sssp_csr(g: OnedGraph, small: bool = False):
    """(row starts, column, weights, light counts, tiny counts, perm, inv)
    the SSSP entry points are given: the renumbered copy for the grid
    search, the split copy in the caller's numbering for the one-block
    search of a small component (it touches a handful of vertices, so the
    numbering buys nothing there and its mapping would add dependent loads
    to a search that takes microseconds)."""
    if g.sr is not None and not small:
        r = g.sr
        return r.rowstarts, r.col, r.w, r.light_deg, r.tiny_deg, r.perm, r.inv
    return g.rowstarts, g.sssp_col, g.sssp_w, g.light_deg, g.tiny_deg, None, None


def _sorted_work(n: int, e: int, dev, bfs_order: bool = False) -> torch.Tensor:
    """Scratch of the canonical build (and of g5_csr_degree_order, which
    needs a little more, when bfs_order)."""
    nb = C.c_uint64()
    _check((lib.g5_csr_degree_order_workspace_size if bfs_order else lib.g5_csr_sorted_workspace_size)(
        n, e, C.byref(nb)))
    return _workspace(nb.value, dev)


def oned_graph_bfs_order(g: OnedGraph, stream=None, work: torch.Tensor | None = None) -> OnedGraph:
    """Gives the BFS its own copy of the column with every row's neighbours
    by decreasing degree (g5_csr_degree_order; col itself, the CSR the
    validators and the reference API see, keeps its canonical order).
    Costs 4 bytes per CSR entry; BFS depths are unchanged (the parents are
    other tree edges of the same graph).  `work`: scratch of at least
    g5_csr_degree_order_workspace_size bytes, else one is allocated."""
    n, e = g.nglobalverts, g.nlocaledges
    nb = C.c_uint64()
    _check(lib.g5_csr_degree_order_workspace_size(n, e, C.byref(nb)))
    if work is None or work.numel() < nb.value:
        work = _workspace(nb.value, g.device)
    bcol = torch.empty(max(e, 1), dtype=torch.int32, device=g.device)
    _check(lib.g5_csr_degree_order(_ptr(g.rowstarts), _ptr(g.col), n, e, _ptr(bcol), _ptr(work), work.numel(),
                                   _stream(stream)))
    btop = torch.empty(max(n, 1), dtype=torch.int32, device=g.device)
    _check(lib.g5_bfs_first_neighbours(_ptr(g.rowstarts), _ptr(bcol), n, _ptr(btop), _stream(stream)))
    g.bcol, g.btop = bcol, btop
    return g


def _bfs_p(g: OnedGraph, params: "BfsParams | None") -> "BfsParams | None":
    """params for a search on g.bfs_col, with the graph's first-neighbour
    array when it has one (a copy: the caller's struct is left alone)."""
    if g.btop is None or g.bcol is None:
        return params
    q = BfsParams(14.0, 24.0, 0, 0) if params is None else BfsParams.from_buffer_copy(params)
    q.top = g.btop.data_ptr()
    return q


def _finish_graph(n, e, rowstarts, col, w, col64, light_delta, work, dedupe, st, dev, stream,
                  with_main, bfs_order, sssp_renumber=True) -> OnedGraph:
    """Canonical rows (already sorted) -> optional dedupe -> the SSSP copy
    (g5_csr_split_light) -> the BFS copy (g5_csr_degree_order, when
    bfs_order) -> isolated bitmap and main component."""
    if dedupe:
        rs2 = torch.empty(n + 1, dtype=torch.int64, device=dev)
        e2 = C.c_uint64()
        _check(lib.g5_csr_dedupe_count(_ptr(rowstarts), _ptr(col), n, e, _ptr(rs2), _ptr(work), work.numel(),
                                       C.byref(e2), st))
        e2 = e2.value
        col2 = torch.empty(max(e2, 1), dtype=torch.int32, device=dev)
        w2 = torch.empty(max(e2, 1), dtype=torch.float32, device=dev)
        c64 = torch.empty(max(e2, 1), dtype=torch.int64, device=dev) if col64 is not None else None
        if e:
            _check(lib.g5_csr_dedupe_copy(_ptr(rowstarts), _ptr(col), _ptr(w), n, _ptr(rs2), _ptr(col2), _ptr(w2),
                                          _ptr(c64), st))
        else:
            rs2.zero_()
        rowstarts, col, w, col64, e = rs2, col2, w2, c64, e2
    scol = torch.empty(max(e, 1), dtype=torch.int32, device=dev)
    sw = torch.empty(max(e, 1), dtype=torch.float32, device=dev)
    light = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    tiny = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    _check(lib.g5_csr_split_light(_ptr(rowstarts), _ptr(col), _ptr(w), n, e, light_delta, _ptr(scol), _ptr(sw),
                                  _ptr(light), _ptr(tiny), _ptr(work), work.numel(), st))
    iso = torch.empty((n + 31) // 32, dtype=torch.int32, device=dev)
    _check(lib.g5_graph_isolated_bitmap(_ptr(rowstarts), n, _ptr(iso), st))
    g = OnedGraph(n, e, rowstarts, col[:e], w[:e], light[:n], light_delta, None if col64 is None else col64[:e], iso)
    g.tiny_deg = tiny[:n]
    g.scol, g.sw = scol[:e], sw[:e]
    if bfs_order:
        oned_graph_bfs_order(g, stream, work)
    if sssp_renumber:
        del work
        oned_graph_sssp_renumber(g, stream)
    if with_main:
        g.main_bits = main_component_bitmap(g, stream)
    return g


def oned_graph_from_tuple_graph(tg: TupleGraph, nglobalverts: int, light_delta: float = 0.1,
                                with_column64: bool = False, stream=None, with_main: bool = True,
                                dedupe: bool = False, bfs_order: bool = True, sssp_renumber: bool = True,
                                radix: bool = True) -> OnedGraph:
    """oned_graph_from_tuple_graph (src/traversal.h:43): the CSR of both
    directions of every non-loop edge, duplicates kept, every row in
    canonical order (sorted by neighbour, then weight bits), plus the SSSP
    copy with light-first rows (g.scol / g.sw, g5_csr_split_light).  The
    rows come from one LSD radix sort of all entries (g5_csr_radix_count +
    g5_csr_radix_fill); radix=False builds the same CSR by degree count,
    source partitioning and row sorts (g5_csr_count + g5_csr_fill_sorted),
    which needs half the scratch.  dedupe=True keeps one entry per (row,
    neighbour), the lightest (not the reference's CSR: its TEPS edge counts
    include duplicates).  with_main=False skips the main-component search
    (g.main_bits = None; set it later with main_component_bitmap).
    bfs_order=False skips the BFS's degree-ordered copy of the column
    (g.bcol; oned_graph_bfs_order makes it later), sssp_renumber=False the
    SSSP's renumbered copy (g.sr; oned_graph_sssp_renumber)."""
    dev = tg.edges.device
    n, m = int(nglobalverts), tg.edges_size
    st = _stream(stream)
    rowstarts = torch.empty(n + 1, dtype=torch.int64, device=dev)
    nent = C.c_uint64()
    if radix:
        nb, ns = C.c_uint64(), C.c_uint64()
        _check(lib.g5_csr_radix_workspace_size(n, m, C.byref(nb)))
        _check((lib.g5_csr_degree_order_workspace_size if bfs_order else lib.g5_csr_sorted_workspace_size)(
            n, 2 * m, C.byref(ns)))
        work = _workspace(max(nb.value, ns.value), dev)
        _check(lib.g5_csr_radix_count(_ptr(tg.edges), m, n, _ptr(work), work.numel(), C.byref(nent), st))
    else:
        nb = C.c_uint64()
        _check(lib.g5_csr_workspace_size(n, m, C.byref(nb)))
        cwork = _workspace(nb.value, dev)
        _check(lib.g5_csr_count(_ptr(tg.edges), m, n, _ptr(rowstarts), _ptr(cwork), cwork.numel(),
                                C.byref(nent), st))
        del cwork
    e = nent.value
    col = torch.empty(max(e, 1), dtype=torch.int32, device=dev)
    w = torch.empty(max(e, 1), dtype=torch.float32, device=dev)
    col64 = torch.empty(max(e, 1), dtype=torch.int64, device=dev) if with_column64 else None
    if radix:
        _check(lib.g5_csr_radix_fill(_ptr(tg.edges), _ptr(tg.weights), m, n, e, _ptr(work), work.numel(),
                                     _ptr(rowstarts), _ptr(col), _ptr(w), _ptr(col64), st))
    else:
        work = _sorted_work(n, e, dev, bfs_order)
        _check(lib.g5_csr_fill_sorted(_ptr(tg.edges), _ptr(tg.weights), m, n, _ptr(rowstarts), e, _ptr(work),
                                      work.numel(), _ptr(col), _ptr(w), _ptr(col64), st))
    return _finish_graph(n, e, rowstarts, col, w, col64, light_delta, work, dedupe, st, dev, stream, with_main,
                         bfs_order, sssp_renumber)


def _split_tiny(rowstarts, col, w, col64, light, n: int, light_delta: float, st) -> torch.Tensor:
    """g5_csr_split_tiny: tiny-first light parts and their tiny counts."""
    tiny = torch.empty(max(n, 1), dtype=torch.int32, device=rowstarts.device)
    _check(lib.g5_csr_split_tiny(_ptr(rowstarts), _ptr(col), _ptr(w), _ptr(col64), _ptr(light), n, light_delta,
                                 _ptr(tiny), st))
    return tiny[:n]


def oned_graph_from_kronecker(seed, log_n: int, nedges: int, device="cuda", light_delta: float = 0.1,
                              with_column64: bool = False, stream=None, with_main: bool = True,
                              dedupe: bool = False, bfs_order: bool = True, sssp_renumber: bool = True) -> OnedGraph:
    """generate_kronecker_range + oned_graph_from_tuple_graph in one step,
    with the generator fused into the CSR passes (no edge list in memory);
    rows then sorted into canonical order (g5_csr_sort_rows) -- the same
    graph as the two-step build.  with_main=False skips the main-component
    search (g.main_bits = None)."""
    n = 1 << log_n
    s = (C.c_uint32 * 5)(*seed)
    nb = C.c_uint64()
    _check(lib.g5_csr_workspace_size(n, nedges, C.byref(nb)))
    cwork = _workspace(nb.value, device)
    rowstarts = torch.empty(n + 1, dtype=torch.int64, device=device)
    nent = C.c_uint64()
    st = _stream(stream)
    _check(lib.g5_csr_count_kronecker(s, log_n, nedges, _ptr(rowstarts), _ptr(cwork), cwork.numel(), C.byref(nent),
                                      st))
    e = nent.value
    col = torch.empty(max(e, 1), dtype=torch.int32, device=device)
    w = torch.empty(max(e, 1), dtype=torch.float32, device=device)
    light = torch.empty(n, dtype=torch.int32, device=device)
    col64 = torch.empty(max(e, 1), dtype=torch.int64, device=device) if with_column64 else None
    # every entry "light" (from the row start): the rows are sorted next
    _check(lib.g5_csr_fill_kronecker(s, log_n, nedges, _ptr(rowstarts), float("inf"), _ptr(cwork), cwork.numel(),
                                     _ptr(col), _ptr(w), None, _ptr(light), st))
    del cwork, light
    work = _sorted_work(n, e, device, bfs_order)
    _check(lib.g5_csr_sort_rows(_ptr(rowstarts), n, e, _ptr(col), _ptr(w), _ptr(col64), _ptr(work), work.numel(),
                                st))
    return _finish_graph(n, e, rowstarts, col, w, col64, light_delta, work, dedupe, st, device, stream, with_main,
                         bfs_order, sssp_renumber)


# ------------------------------------------------------- packed graphs ----

class PackedGraphs:
    """Disjoint graphs packed into one CSR (g5_csr_pack_append): graph i
    owns vertices [vbase[i], vbase[i] + nverts[i]) and the entries of their
    rows; `g` is the union as an OnedGraph.  One root per graph then makes a
    single g5_bfs_traverse_multi / g5_sssp_traverse_multi launch compute
    every graph's own BFS / SSSP (no counterpart in the reference, which
    holds one graph)."""

    def __init__(self, nverts, vbase, g: OnedGraph, roots):
        self.nverts = np.asarray(nverts, np.int64)
        self.vbase = np.asarray(vbase, np.int64)
        self.g = g
        self.local_roots = np.asarray(roots, np.int64)
        self.roots = self.vbase + self.local_roots
        self.d_roots = torch.as_tensor(self.roots, dtype=torch.int64, device=g.device)

    @property
    def ngraphs(self) -> int:
        return len(self.vbase)

    def graph_slice(self, i: int) -> slice:
        return slice(int(self.vbase[i]), int(self.vbase[i] + self.nverts[i]))


def pack_graphs(graphs, roots, device="cuda", stream=None, sssp_renumber: bool = True) -> PackedGraphs:
    """Packs the OnedGraphs in `graphs`; roots[i] is graph i's root (its own
    vertex number).  pack_kronecker builds and packs generated graphs one
    at a time instead, without holding them all unpacked.  sssp_renumber:
    the union also gets the SSSP's renumbered copy (oned_graph_sssp_renumber)."""
    graphs = list(graphs)
    sizes = [(g.nglobalverts, g.nlocaledges) for g in graphs]
    return _pack(sizes, iter(graphs), roots, device, graphs[0].light_delta if graphs else 0.1, stream, sssp_renumber)


def pack_kronecker(scales, edgefactor: int = 16, seed1_base: int = 2, seed2: int = 3, device="cuda",
                   light_delta: float = 0.1, stream=None, sssp_renumber: bool = True) -> PackedGraphs:
    """Generates Kronecker graph i (SCALE scales[i], seeds (seed1_base + i,
    seed2)) with the fused generator -> CSR path and packs it at once; each
    graph's root is its first Graph500 root (the runner's choice)."""
    scales = [int(x) for x in scales]
    # Entries are at most 2 per edge (self-loops store one): size for that.
    sizes = [(1 << s, 2 * edgefactor << s) for s in scales]
    roots: list[int] = []

    def gen():
        for i, s in enumerate(scales):
            g = oned_graph_from_kronecker(make_mrg_seed(seed1_base + i, seed2), s, edgefactor << s, device=device,
                                          light_delta=light_delta, stream=stream, with_main=False, bfs_order=False,
                                          sssp_renumber=False)
            r = generate_bfs_roots(g, 2, 3, 1)
            roots.append(r[0] if r else 0)
            yield g

    return _pack(sizes, gen(), roots, device, light_delta, stream, sssp_renumber)


def _pack(sizes, graphs, roots, device, light_delta, stream, sssp_renumber=True) -> PackedGraphs:
    N = sum(n for n, _ in sizes)
    Emax = sum(e for _, e in sizes)
    if N > (1 << 31):
        raise ValueError(f"pack: {N} vertices exceed 2^31")
    rowstarts = torch.empty(N + 1, dtype=torch.int64, device=device)
    col = torch.empty(max(Emax, 1), dtype=torch.int32, device=device)
    w = torch.empty(max(Emax, 1), dtype=torch.float32, device=device)
    light = torch.empty(max(N, 1), dtype=torch.int32, device=device)
    st = _stream(stream)
    vb, eb = 0, 0
    nverts, vbase = [], []
    for g in graphs:
        _check(lib.g5_csr_pack_append(_ptr(g.rowstarts), _ptr(g.sssp_col), _ptr(g.sssp_w), _ptr(g.light_deg),
                                      g.nglobalverts,
                                      g.nlocaledges, vb, eb, _ptr(rowstarts), _ptr(col), _ptr(w), _ptr(light), st))
        nverts.append(g.nglobalverts)
        vbase.append(vb)
        vb += g.nglobalverts
        eb += g.nlocaledges
        del g
    if vb == 0:
        raise ValueError("pack: no graphs")
    iso = torch.empty((vb + 31) // 32, dtype=torch.int32, device=device)
    _check(lib.g5_graph_isolated_bitmap(_ptr(rowstarts), vb, _ptr(iso), st))
    u = OnedGraph(vb, eb, rowstarts[:vb + 1], col[:eb], w[:eb], light[:vb], light_delta, None, iso)
    # Packed rows keep their order; the split (a no-op on split rows) yields
    # the packed graph's tiny counts.
    u.tiny_deg = _split_tiny(u.rowstarts, u.col, u.w, None, u.light_deg, vb, light_delta, st)
    if sssp_renumber:
        oned_graph_sssp_renumber(u, stream)
    return PackedGraphs(nverts, vbase, u, list(roots))


def oned_graph_bfs_traverse_multi(g: OnedGraph, bfs: "BfsState", d_roots: torch.Tensor, params=None,
                                  with_depth: bool = True, stream=None) -> None:
    """BFS from every root in d_roots (device int64) at once
    (g5_bfs_traverse_multi); reset bfs first."""
    params = _bfs_p(g, params)
    _check(lib.g5_bfs_traverse_multi(_ptr(g.rowstarts), _ptr(g.bfs_col), g.nglobalverts, _ptr(d_roots), d_roots.numel(),
                                     _ptr(bfs.pred), _ptr(bfs.depth) if with_depth else None, _ptr(bfs.work),
                                     bfs.work.numel(), C.byref(params) if params is not None else None,
                                     _stream(stream)))


def oned_graph_sssp_traverse_multi(g: OnedGraph, sssp: "SsspState", d_roots: torch.Tensor, delta: float = 0.1,
                                   blocks: int = 0, pull: float = 0.0, sub_min: int = 0, stream=None,
                                   big_deg: int = 0, chunk: int = 0) -> None:
    """SSSP from every source in d_roots at once (g5_sssp_traverse_multi);
    reset sssp first."""
    rs, col, w, light, tiny, perm, inv = _sssp_csr(g)
    p = SsspParams(delta, blocks, pull, sub_min, 0, _ptr(tiny), 0, big_deg, chunk, _ptr(perm), _ptr(inv))
    _check(lib.g5_sssp_traverse_multi(_ptr(rs), _ptr(col), _ptr(w), _ptr(light),
                                      g.light_delta,
                                      g.nglobalverts, _ptr(d_roots), d_roots.numel(), _ptr(sssp.dist),
                                      _ptr(sssp.pred), _ptr(sssp.work), sssp.work.numel(), C.byref(p),
                                      _stream(stream)))


class PackedBatch:
    """One BFS and one SSSP from every packed graph's root: reset, the
    multi-root BFS, reset, the multi-source SSSP -- four library calls on one
    stream, captured once into a CUDA graph and replayed per batch (no
    per-graph launches, no host work between them)."""

    def __init__(self, pk: PackedGraphs, delta: float = 0.1, capture: bool = True, with_depth: bool = True,
                 bfs_params: BfsParams | None = None, sssp_blocks: int = 0, sssp_pull: float = 0.0,
                 sssp_sub_min: int = 0, sssp_big_deg: int = 0, sssp_chunk: int = 0):
        self.pk, self.delta, self.with_depth = pk, delta, with_depth
        self.bfs_params, self.sssp_blocks = bfs_params, sssp_blocks
        self.sssp_pull, self.sssp_sub_min = sssp_pull, sssp_sub_min
        self.sssp_big_deg, self.sssp_chunk = sssp_big_deg, sssp_chunk
        self.bfs = BfsState(pk.g)
        self.sssp = SsspState(pk.g)
        self.stream = torch.cuda.Stream(device=pk.g.device)
        self.graph = None
        # One eager batch first: the library's once-per-device setup (L2
        # window, occupancy queries) must not happen inside the capture.
        self.run()
        self.stream.synchronize()
        if capture:
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph, stream=self.stream):
                self._enqueue_bfs()
                self._enqueue_sssp()

    def _enqueue_bfs(self):
        oned_graph_bfs_reset(self.bfs, self.with_depth, self.pk.g)
        oned_graph_bfs_traverse_multi(self.pk.g, self.bfs, self.pk.d_roots, self.bfs_params,
                                      with_depth=self.with_depth)

    def _enqueue_sssp(self):
        oned_graph_sssp_reset(self.sssp)
        oned_graph_sssp_traverse_multi(self.pk.g, self.sssp, self.pk.d_roots, self.delta, self.sssp_blocks,
                                       self.sssp_pull, self.sssp_sub_min, big_deg=self.sssp_big_deg,
                                       chunk=self.sssp_chunk)

    def run(self) -> None:
        """Enqueues one batch on self.stream (replaying the graph when captured)."""
        with torch.cuda.stream(self.stream):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._enqueue_bfs()
                self._enqueue_sssp()

    def check(self) -> None:
        """Raises if either search of the last batch reported a device error."""
        bfs_stats(self.bfs, self.stream)
        sssp_status(self.sssp, self.stream)


def main_component_bitmap(g: OnedGraph, stream=None) -> np.ndarray:
    """Host bitmap of the component of a maximum-degree vertex (the giant
    component of a Kronecker graph): one BFS from it at build time.  Queries
    from roots outside it run on a single block (g5_bfs_query)."""
    if g.nlocaledges == 0:
        return np.zeros((g.nglobalverts + 31) // 32, np.uint32)
    hub = int(torch.argmax(g.rowstarts[1:] - g.rowstarts[:-1]))
    bfs = BfsState(g)
    _check(lib.g5_bfs_reset(g.nglobalverts, _ptr(bfs.pred), None, None, _ptr(bfs.work), bfs.work.numel(),
                            _stream(stream)))
    hp = _bfs_p(g, None)
    _check(lib.g5_bfs_traverse(_ptr(g.rowstarts), _ptr(g.bfs_col), g.nglobalverts, hub, _ptr(bfs.pred), None,
                               _ptr(bfs.work), bfs.work.numel(), C.byref(hp) if hp is not None else None,
                               _stream(stream)))
    bits = torch.empty((g.nglobalverts + 31) // 32, dtype=torch.int32, device=g.device)
    _check(lib.g5_bfs_visited_bitmap(_ptr(bfs.work), bfs.work.numel(), g.nglobalverts, _ptr(bits),
                                     _stream(stream)))
    bfs_stats(bfs, stream)  # surfaces any device error
    return bits.cpu().numpy().view(np.uint32)


def oned_graph_is_vertex_isolated(g: OnedGraph, global_vertex: int) -> bool:
    """oned_graph_is_vertex_isolated (src/traversal.h:44); raises on a vertex
    outside [0, N) where the reference aborts."""
    if not 0 <= global_vertex < g.nglobalverts:
        raise ValueError(f"Vertex {global_vertex} is outside graph vertex range [0, {g.nglobalverts})")
    r = g.rowstarts[global_vertex:global_vertex + 2].cpu()
    return bool(r[0] == r[1])


def generate_bfs_roots(g: OnedGraph, seed1: int = 2, seed2: int = 3, max_roots: int = 64) -> list[int]:
    """Root choice of the runner's generate_bfs_roots
    (examples/graph500_runner.cu:43-74): up to max_roots distinct vertices of
    nonzero degree from the seeded MRG doubles."""
    n = g.nglobalverts
    deg0 = (g.rowstarts[1:] == g.rowstarts[:-1]).cpu().numpy()
    roots: list[int] = []
    counter = 0
    while len(roots) < max_roots:
        found = False
        while True:
            d = make_random_numbers(2, seed1, seed2, counter)
            root = int(np.uint64((d[0] + d[1]) * float(n))) % n
            counter += 2
            if counter > 2 * n:
                break
            if root in roots or deg0[root]:
                continue
            found = True
            break
        if not found:
            break
        roots.append(root)
    return roots


# ----------------------------------------------------------------- BFS ----

def bfs_workspace_bytes(nverts: int) -> int:
    """Bytes of the BFS workspace for a graph of nverts vertices
    (g5_bfs_workspace_size)."""
    nb = C.c_uint64()
    _check(lib.g5_bfs_workspace_size(nverts, C.byref(nb)))
    return nb.value


class BfsState:
    """Bfs_State (src/traversal.h:18-28): pred int64[N], depth int32[N],
    dist int64[N] (filled by bfs_compute_dist_from_pred) and the kernel's
    workspace."""

    def __init__(self, g: OnedGraph):
        n = g.nglobalverts
        dev = g.device
        nb = C.c_uint64()
        _check(lib.g5_bfs_workspace_size(n, C.byref(nb)))
        self.work = _workspace(nb.value, dev)
        self.pred = torch.empty(n, dtype=torch.int64, device=dev)
        self.depth = torch.empty(n, dtype=torch.int32, device=dev)
        self.dist: torch.Tensor | None = None
        self.val_work: torch.Tensor | None = None
        self.max_nlocalverts = n
        # After its first reset the state undoes only what each search
        # wrote (g5_bfs_reset_touched); the first one clears everything.
        self.was_reset = False
        # Pinned: the query path's kernel writes the statistics here itself.
        self._h_stats_buf = torch.zeros(C.sizeof(BfsStats), dtype=torch.uint8).pin_memory()
        self.h_stats = BfsStats.from_address(self._h_stats_buf.data_ptr())
        self._plan = None  # (graph, with_depth, stream, g5_bfs_query_plan*, main bitmap) of the query path

    def drop_plan(self) -> None:
        if self._plan is not None:
            lib.g5_bfs_query_plan_destroy(self._plan[3])
            self._plan = None

    def __del__(self):
        try:
            self.drop_plan()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass


def oned_graph_bfs_create(g: OnedGraph) -> BfsState:
    return BfsState(g)


def oned_graph_bfs_run(g: OnedGraph, bfs: BfsState, root: int, params: BfsParams | None = None,
                       with_depth: bool = True, stream=None) -> None:
    """oned_graph_bfs_run (src/traversal.h:47) with its clear: enqueues the
    whole BFS (reset + persistent kernel)."""
    oned_graph_bfs_reset(bfs, with_depth, g, stream)
    oned_graph_bfs_traverse(g, bfs, root, params, with_depth, stream)


def oned_graph_bfs_reset(bfs: BfsState, with_depth: bool = True, g: OnedGraph | None = None,
                         stream=None) -> None:
    """First half of oned_graph_bfs_run (the reference's oned_graph_bfs_clear):
    clear pred/depth and the workspace; with the graph, isolated vertices
    start out visited.  After the state's first reset only what the last
    search wrote is undone (O(reached) after a one-block search)."""
    fn = lib.g5_bfs_reset_touched if bfs.was_reset else lib.g5_bfs_reset
    _check(fn(bfs.max_nlocalverts, _ptr(bfs.pred), _ptr(bfs.depth) if with_depth else None,
              _ptr(g.isolated) if g is not None else None, _ptr(bfs.work), bfs.work.numel(), _stream(stream)))
    bfs.was_reset = True


def _right_sized(g: OnedGraph, root: int, params: BfsParams | None) -> BfsParams | None:
    if params is None and not g.in_main_component(root):
        return BfsParams(14.0, 24.0, 3, 1)  # small component: the lean one-block search
    return params


def oned_graph_bfs_traverse(g: OnedGraph, bfs: BfsState, root: int, params: BfsParams | None = None,
                            with_depth: bool = True, stream=None) -> None:
    """Second half of oned_graph_bfs_run: the persistent BFS kernel alone
    (one block for a root outside the main component)."""
    params = _bfs_p(g, _right_sized(g, root, params))
    _check(lib.g5_bfs_traverse(_ptr(g.rowstarts), _ptr(g.bfs_col), g.nglobalverts, root, _ptr(bfs.pred),
                               _ptr(bfs.depth) if with_depth else None, _ptr(bfs.work), bfs.work.numel(),
                               C.byref(params) if params is not None else None, _stream(stream)))


def _main_bits_ptr(g: OnedGraph) -> int | None:
    """Host address of g.main_bits, looked up once per array."""
    mb = g.main_bits
    if mb is None:
        return None
    c = g.__dict__.get("_main_bits_addr")
    if c is None or c[0] is not mb:
        c = (mb, mb.ctypes.data)
        g.__dict__["_main_bits_addr"] = c
    return c[1]


# One record of g5_bfs_export.
REACHED_DTYPE = np.dtype([("vertex", "<u4"), ("depth", "<i4"), ("parent", "<i8")])


def oned_graph_bfs_export(g: OnedGraph, bfs: BfsState, with_depth: bool = False, stream=None,
                          out: torch.Tensor | None = None) -> np.ndarray | torch.Tensor:
    """The last search's result for the host (g5_bfs_export): one record
    (vertex, depth, parent) per reached vertex, root included -- depth -1
    unless with_depth (the search must have kept depths: a query or run
    with_depth).  `out`: a uint8 tensor of at least 16 bytes per record, in
    pinned host memory (the kernel writes the records there itself; the
    result is a numpy structured view of REACHED_DTYPE) or on the device (a
    byte tensor of the records); by default a pinned buffer of the state,
    overwritten by its next export.  After a one-block search the records
    come from its touched list, in the order reached (the cost follows the
    result); otherwise in no particular order."""
    n = g.nglobalverts
    if out is None:
        if getattr(bfs, "_xbuf", None) is None or bfs._xbuf.numel() < 16 * n:
            bfs._xbuf = torch.empty(16 * n, dtype=torch.uint8).pin_memory()
        out = bfs._xbuf
    if getattr(bfs, "_xcnt", None) is None:
        bfs._xcnt = torch.zeros(8, dtype=torch.uint8).pin_memory()
    cap = out.numel() // 16
    _check(lib.g5_bfs_export(_ptr(bfs.pred), _ptr(bfs.depth) if with_depth else None, n, _ptr(bfs.work),
                             bfs.work.numel(), _ptr(out), cap, bfs._xcnt.data_ptr(), _stream(stream)))
    cnt = int(C.c_uint64.from_address(bfs._xcnt.data_ptr()).value)
    if out.device.type == "cpu":
        return out.numpy()[: 16 * cnt].view(REACHED_DTYPE)
    return out[: 16 * cnt]


def oned_graph_bfs_query(g: OnedGraph, bfs: BfsState, root: int, with_depth: bool = False,
                         stream=None, params: BfsParams | None = None) -> BfsStats:
    """One search end to end from the host, the reference's synchronous
    oned_graph_bfs_run on a state reset since its last search: the root goes
    to the device as a launch argument, the device writes the statistics to
    pinned host memory, and the host waits on them.  Runs through a
    g5_bfs_query_plan made on the first query of this state with this graph,
    depth choice, stream and params (C ABI: two arguments per query); with
    params.blocks == 0 a root outside the main component still gets the
    one-block search."""
    st = _stream(stream)
    plan = bfs._plan
    if (plan is None or plan[0] is not g or plan[1] != with_depth or plan[2] != st or plan[4] is not g.main_bits
            or plan[5] is not params or plan[6] is not g.bfs_col):
        plan = _make_query_plan(g, bfs, with_depth, st, params)
    rc = _plan_run(plan[3], root)
    if rc:
        _check(rc)
    return bfs.h_stats


def oned_graph_bfs_query_export(g: OnedGraph, bfs: BfsState, root: int, with_depth: bool = True,
                                out: torch.Tensor | None = None, stream=None,
                                params: BfsParams | None = None) -> tuple[BfsStats, np.ndarray]:
    """oned_graph_bfs_query and oned_graph_bfs_export in one C call
    (g5_bfs_query_plan_export): the search, then right behind it in the
    stream the export of its result into pinned host memory (`out`, a
    pinned uint8 tensor of 16 bytes a record; by default the state's own
    buffer), with one wait on the host.  Returns the statistics and the
    records (REACHED_DTYPE, a view of `out`)."""
    st = _stream(stream)
    plan = bfs._plan
    if (plan is None or plan[0] is not g or plan[1] != with_depth or plan[2] != st or plan[4] is not g.main_bits
            or plan[5] is not params or plan[6] is not g.bfs_col):
        plan = _make_query_plan(g, bfs, with_depth, st, params)
    if out is None:
        if getattr(bfs, "_xbuf", None) is None or bfs._xbuf.numel() < 16 * g.nglobalverts:
            bfs._xbuf = torch.empty(16 * g.nglobalverts, dtype=torch.uint8).pin_memory()
        out = bfs._xbuf
    if getattr(bfs, "_xcnt", None) is None:
        bfs._xcnt = torch.zeros(8, dtype=torch.uint8).pin_memory()
    rc = _plan_export(plan[3], root, out.data_ptr(), out.numel() // 16, bfs._xcnt.data_ptr())
    if rc:
        _check(rc)
    cnt = int(C.c_uint64.from_address(bfs._xcnt.data_ptr()).value)
    return bfs.h_stats, out.numpy()[: 16 * cnt].view(REACHED_DTYPE)


def _make_query_plan(g: OnedGraph, bfs: BfsState, with_depth: bool, st, params: BfsParams | None = None):
    bfs.drop_plan()
    h = C.c_void_p()
    cp = _bfs_p(g, params)  # the plan copies it
    _check(lib.g5_bfs_query_plan_create(g.rowstarts.data_ptr(), g.bfs_col.data_ptr(), g.nglobalverts, _main_bits_ptr(g),
                                        bfs.pred.data_ptr(), bfs.depth.data_ptr() if with_depth else None,
                                        bfs.work.data_ptr(), bfs.work.numel(),
                                        C.byref(cp) if cp is not None else None, C.byref(bfs.h_stats), st,
                                        C.byref(h)))
    # The graph (and params) are held with the plan: the plan keeps its device pointers.
    bfs._plan = (g, with_depth, st, h.value, g.main_bits, params, g.bfs_col)
    return bfs._plan


def bfs_stats(bfs: BfsState, stream=None) -> BfsStats:
    s = BfsStats()
    _check(lib.g5_bfs_last_stats(_ptr(bfs.work), bfs.work.numel(), C.byref(s), _stream(stream)))
    return s


def bfs_trace(bfs: BfsState, stream=None) -> dict:
    """Per-level trace of the last BFS on this state (direction, frontier
    size and edges, device milliseconds)."""
    k = 64
    mode = np.zeros(k, np.int32)
    nv = np.zeros(k, np.uint64)
    ne = np.zeros(k, np.uint64)
    ms = np.zeros(k, np.float64)
    nl, solo = C.c_int32(), C.c_int32()
    _check(lib.g5_bfs_last_trace(_ptr(bfs.work), bfs.work.numel(), k, mode.ctypes.data, nv.ctypes.data,
                                 ne.ctypes.data, ms.ctypes.data, C.byref(nl), C.byref(solo), _stream(stream)))
    n = min(nl.value, k)
    return {"levels": nl.value, "solo_levels": solo.value, "mode": mode[:n].tolist(),
            "frontier": nv[:n].tolist(), "frontier_edges": ne[:n].tolist(), "ms": ms[:n].tolist()}


def bfs_compute_dist_from_pred(g: OnedGraph, bfs: BfsState, root: int, stream=None) -> torch.Tensor:
    """bfs_compute_dist_from_pred (src/traversal.h:48)."""
    if bfs.dist is None:
        bfs.dist = torch.empty(g.nglobalverts, dtype=torch.int64, device=g.device)
    if bfs.val_work is None:
        bfs.val_work = _val_work(g)
    _check(lib.g5_bfs_dist_from_pred(_ptr(g.rowstarts), _ptr(g.col), g.nglobalverts, _ptr(bfs.pred), root,
                                     _ptr(bfs.dist), _ptr(bfs.val_work), bfs.val_work.numel(), _stream(stream)))
    return bfs.dist


# --------------------------------------------------------- batched BFS ----

MSBFS_MAX_ROOTS = 256


class MsBfsState:
    """Workspace of the batched BFS (g5_msbfs_*) bound to one graph: up to
    256 roots per search, one bit each.  No counterpart in the reference,
    which runs oned_graph_bfs_run once per root (src/traversal.h:47)."""

    def __init__(self, g: OnedGraph, depth_bits: int = 0, stream=None):
        self.n = g.nglobalverts
        self.nentries = g.nlocaledges
        self.depth_bits = depth_bits
        nb = C.c_uint64()
        _check(lib.g5_msbfs_workspace_size(self.n, self.nentries, depth_bits, C.byref(nb)))
        self.work = _workspace(nb.value, g.device)
        self.nroots = 0
        self.h_roots = torch.zeros(MSBFS_MAX_ROOTS, dtype=torch.int64).pin_memory()
        _check(lib.g5_msbfs_prepare(_ptr(g.rowstarts), _ptr(g.col), self.n, self.nentries, depth_bits,
                                    _ptr(self.work), self.work.numel(), _stream(stream)))


def msbfs_run(g: OnedGraph, ms: MsBfsState, roots, params: MsBfsParams | None = None, sync: bool = True,
              stream=None) -> MsBfsStats | None:
    """Searches from every root in `roots` (1..256 vertex ids) at once on
    the graph `ms` was prepared for (its own copy of g).  With sync, waits
    and returns the statistics (raising on a failed search); otherwise only
    enqueues."""
    roots = [int(r) for r in roots]
    if not 1 <= len(roots) <= MSBFS_MAX_ROOTS:
        raise ValueError(f"msbfs_run: {len(roots)} roots, expected 1..{MSBFS_MAX_ROOTS}")
    ms.h_roots[:len(roots)] = torch.tensor(roots, dtype=torch.int64)
    ms.nroots = len(roots)
    st = MsBfsStats() if sync else None
    _check(lib.g5_msbfs_run(ms.n, ms.nentries, ms.depth_bits, ms.h_roots.data_ptr(), len(roots),
                            _ptr(ms.work), ms.work.numel(),
                            C.byref(params) if params is not None else None,
                            C.byref(st) if st is not None else None, _stream(stream)))
    return st


def msbfs_depths_u8(ms: MsBfsState, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Depths of the last search, uint8[nroots, N] (255 = not reached)."""
    if out is None:
        out = torch.empty((ms.nroots, ms.n), dtype=torch.uint8, device=ms.work.device)
    _check(lib.g5_msbfs_depths_u8(_ptr(ms.work), ms.work.numel(), ms.n, ms.nentries, ms.depth_bits, ms.nroots,
                                  _ptr(out), _stream(stream)))
    return out


def msbfs_depth(ms: MsBfsState, root_index: int, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Root `root_index`'s depth array, int32[N] with -1 where unreached (the
    layout of BfsState.depth)."""
    if out is None:
        out = torch.empty(ms.n, dtype=torch.int32, device=ms.work.device)
    _check(lib.g5_msbfs_depth(_ptr(ms.work), ms.work.numel(), ms.n, ms.nentries, ms.depth_bits, root_index,
                              _ptr(out), _stream(stream)))
    return out


def msbfs_stats(ms: MsBfsState, stream=None) -> MsBfsStats:
    s = MsBfsStats()
    _check(lib.g5_msbfs_last_stats(_ptr(ms.work), ms.work.numel(), C.byref(s), _stream(stream)))
    return s


def msbfs_trace(ms: MsBfsState, stream=None) -> dict:
    k = 64
    mode = np.zeros(k, np.int32)
    nv = np.zeros(k, np.uint64)
    ne = np.zeros(k, np.uint64)
    tm = np.zeros(k, np.float64)
    nl = C.c_int32()
    _check(lib.g5_msbfs_last_trace(_ptr(ms.work), ms.work.numel(), k, mode.ctypes.data, nv.ctypes.data,
                                   ne.ctypes.data, tm.ctypes.data, C.byref(nl), _stream(stream)))
    n = min(nl.value, k)
    return {"levels": nl.value, "mode": mode[:n].tolist(), "frontier": nv[:n].tolist(),
            "frontier_edges": ne[:n].tolist(), "ms": tm[:n].tolist()}


# ---------------------------------------------------------------- SSSP ----

def sssp_workspace_bytes(nverts: int) -> int:
    """Bytes of the SSSP workspace for a graph of nverts vertices
    (g5_sssp_workspace_size)."""
    nb = C.c_uint64()
    _check(lib.g5_sssp_workspace_size(nverts, C.byref(nb)))
    return nb.value


class SsspState:
    """Sssp_State (src/traversal.h:30-41): pred int64[N], dist float32[N]."""

    def __init__(self, g: OnedGraph):
        n = g.nglobalverts
        dev = g.device
        nb = C.c_uint64()
        _check(lib.g5_sssp_workspace_size(n, C.byref(nb)))
        self.work = _workspace(nb.value, dev)
        self.pred = torch.empty(n, dtype=torch.int64, device=dev)
        self.dist = torch.empty(n, dtype=torch.float32, device=dev)
        self.max_nlocalverts = n
        self.was_reset = False  # later resets undo only what the last search wrote


def oned_graph_sssp_create(g: OnedGraph) -> SsspState:
    return SsspState(g)


def _sssp_params(g: OnedGraph, root: int, delta, blocks, pull, sub_min, small, check_opens=False, big_deg=0,
                 chunk=0) -> SsspParams:
    # small=None: the lean one-block search for a root outside the main
    # component (when the grid is left to the library).
    if small is None:
        small = blocks == 0 and not g.in_main_component(root)
    _, _, _, _, tiny, perm, inv = _sssp_csr(g, bool(small))
    return SsspParams(delta, 1 if small and blocks == 0 else blocks, pull, sub_min, int(bool(small)),
                      _ptr(tiny), int(bool(check_opens)), big_deg, chunk, _ptr(perm), _ptr(inv))


def oned_graph_sssp_run(g: OnedGraph, sssp: SsspState, root: int, delta: float = 0.1, blocks: int = 0,
                        pull: float = 0.0, sub_min: int = 0, small: bool | None = None, stream=None,
                        check_opens: bool = False, big_deg: int = 0, chunk: int = 0) -> None:
    """oned_graph_sssp_run (src/traversal.h:52), delta 0.1 as the reference.
    check_opens: the bucket and sub-bucket opens exchange their stamps and
    fail the search if a queue held a vertex twice (a test aid).  big_deg /
    chunk: the work tiles of g5_sssp_params (0 = defaults)."""
    p = _sssp_params(g, root, delta, blocks, pull, sub_min, small, check_opens, big_deg, chunk)
    rs, col, w, light = _sssp_csr(g, bool(p.small))[:4]
    _check(lib.g5_sssp_run(_ptr(rs), _ptr(col), _ptr(w), _ptr(light), g.light_delta,
                           g.nglobalverts, root, _ptr(sssp.dist), _ptr(sssp.pred), _ptr(sssp.work),
                           sssp.work.numel(), C.byref(p), _stream(stream)))
    sssp.was_reset = True  # g5_sssp_run resets in full first


def sssp_multi_workspace(g: OnedGraph) -> torch.Tensor:
    """Scratch of oned_graph_sssp_multi (about 276 bytes per vertex)."""
    nb = C.c_uint64()
    _check(lib.g5_sssp_multi_workspace_size(g.nglobalverts, C.byref(nb)))
    return _workspace(nb.value, g.device)


class SsspMultiState:
    """A batched-SSSP workspace of one graph with its distance outputs for
    up to 32 sources (dist[s] for source s of the last run)."""

    def __init__(self, g: OnedGraph, max_sources: int = 32):
        self.work = sssp_multi_workspace(g)
        self.dist = torch.empty((max_sources, g.nglobalverts), dtype=torch.float32, device=g.device)
        self.max_sources = max_sources


def sssp_multi_status(state: SsspMultiState, stream=None) -> SsspMultiStats:
    """Statistics of the state's last batched run; raises on a device error
    (synchronises the stream)."""
    st = SsspMultiStats()
    _check(lib.g5_sssp_multi_last_stats(_ptr(state.work), state.work.numel(), C.byref(st), _stream(stream)))
    return st


def oned_graph_sssp_multi(g: OnedGraph, sources, work: torch.Tensor | None = None, with_pred: bool = True,
                          blocks: int = 0, stream=None, delta: float = 0.0, dist: torch.Tensor | None = None,
                          pred: torch.Tensor | None = None,
                          sync: bool = True) -> tuple[torch.Tensor, torch.Tensor | None, SsspMultiStats | None]:
    """SSSP from up to 32 sources of g in one launch (g5_sssp_multi_run):
    dist[s] / pred[s] equal oned_graph_sssp_run's outputs from sources[s]
    bit for bit (float32 distances, -1.0 / -1 where unreached).  Runs on the
    graph's renumbered SSSP copy when it has one (sources and outputs stay
    in the caller's numbering).  delta: the shared bucket width (0 = 0.1;
    results never depend on it).  `work`: sssp_multi_workspace(g), else one
    is allocated; `dist` / `pred`: [len(sources), N] outputs to reuse.
    sync=False: no wait (statistics None; sssp_multi_status reads them)."""
    src = [int(x) for x in sources]
    k, n = len(src), g.nglobalverts
    if work is None:
        work = sssp_multi_workspace(g)
    if dist is None:
        dist = torch.empty((k, n), dtype=torch.float32, device=g.device)
    if with_pred and pred is None:
        pred = torch.empty((k, n), dtype=torch.int64, device=g.device)
    rs, col, w, _, _, perm, inv = _sssp_csr(g)
    h_src = (C.c_uint64 * max(k, 1))(*src)
    st = SsspMultiStats() if sync else None
    _check(lib.g5_sssp_multi_run(_ptr(rs), _ptr(col), _ptr(w), n, _ptr(perm), _ptr(inv), h_src, k, _ptr(dist),
                                 _ptr(pred) if with_pred else None, _ptr(work), work.numel(), delta, blocks,
                                 C.byref(st) if sync else None, _stream(stream)))
    return dist, (pred if with_pred else None), st


def oned_graph_sssp_reset(sssp: SsspState, stream=None) -> None:
    """The reset half of oned_graph_sssp_run (the reference's
    oned_graph_sssp_clear, which its runner keeps outside the timed region):
    workspace cleared, dist = -1.0f and pred = -1 everywhere, so the search
    writes only the vertices it reaches.  After the state's first reset only
    what the last search wrote is undone (O(reached) after a one-block
    search)."""
    fn = lib.g5_sssp_reset_touched if sssp.was_reset else lib.g5_sssp_reset
    _check(fn(sssp.max_nlocalverts, _ptr(sssp.dist), _ptr(sssp.pred), _ptr(sssp.work), sssp.work.numel(),
              _stream(stream)))
    sssp.was_reset = True


def oned_graph_sssp_traverse(g: OnedGraph, sssp: SsspState, root: int, delta: float = 0.1, blocks: int = 0,
                             pull: float = 0.0, sub_min: int = 0, small: bool | None = None,
                             stream=None, check_opens: bool = False, big_deg: int = 0, chunk: int = 0) -> None:
    """The search itself, on a reset state (the lean one-block search for a
    root outside the main component)."""
    p = _sssp_params(g, root, delta, blocks, pull, sub_min, small, check_opens, big_deg, chunk)
    rs, col, w, light = _sssp_csr(g, bool(p.small))[:4]
    _check(lib.g5_sssp_traverse(_ptr(rs), _ptr(col), _ptr(w), _ptr(light),
                                g.light_delta,
                                g.nglobalverts, root, _ptr(sssp.dist), _ptr(sssp.pred), _ptr(sssp.work),
                                sssp.work.numel(), C.byref(p), _stream(stream)))


def sssp_trace(sssp: SsspState, stream=None) -> dict:
    """Counters and per-phase trace of the last SSSP on this state."""
    k = 256
    counts = np.zeros(7, np.uint64)
    kind = np.zeros(k, np.int32)
    size = np.zeros(k, np.uint64)
    ms = np.zeros(k, np.float64)
    edges = np.zeros(k, np.uint64)
    n = C.c_int32()
    _check(lib.g5_sssp_last_trace(_ptr(sssp.work), sssp.work.numel(), counts.ctypes.data, k, kind.ctypes.data,
                                  size.ctypes.data, ms.ctypes.data, edges.ctypes.data, C.byref(n), _stream(stream)))
    m = min(n.value, k)
    names = ["edges", "settled_skips", "atomics", "improved", "ring_pushes", "frontier_pushes", "pulls"]
    return {"counts": dict(zip(names, counts.tolist())), "phases": n.value, "kind": kind[:m].tolist(),
            "size": size[:m].tolist(), "ms": ms[:m].tolist(), "edges": edges[:m].tolist()}


def sssp_status(sssp: SsspState, stream=None) -> tuple[int, int]:
    b, ph = C.c_uint64(), C.c_uint64()
    _check(lib.g5_sssp_last_status(_ptr(sssp.work), sssp.work.numel(), C.byref(b), C.byref(ph),
                                   _stream(stream)))
    return b.value, ph.value


# ---------------------------------------------------------- validation ----

def _val_work(g: OnedGraph) -> torch.Tensor:
    nb = C.c_uint64()
    _check(lib.g5_validate_workspace_size(g.nglobalverts, C.byref(nb)))
    return _workspace(nb.value, g.device)


def edge_count(g: OnedGraph, pred: torch.Tensor, work: torch.Tensor | None = None, stream=None) -> int:
    """oned_graph_edge_count (examples/graph500_runner.cu:184-201)."""
    work = _val_work(g) if work is None else work
    out = C.c_uint64()
    _check(lib.g5_edge_count(_ptr(g.rowstarts), _ptr(g.col), g.nglobalverts, _ptr(pred), _ptr(work),
                             work.numel(), C.byref(out), _stream(stream)))
    return out.value


def bfs_validate(g: OnedGraph, root: int, pred: torch.Tensor, dist: torch.Tensor,
                 work: torch.Tensor | None = None, stream=None) -> int:
    """Error count of oned_graph_bfs_validate (examples/graph500_runner.cu:203-255);
    on the SSSP's renumbered copy when the graph has one (the same count,
    faster: the records the rules read are in degree order)."""
    work = _val_work(g) if work is None else work
    out = C.c_uint64()
    if g.sr is not None:
        _check(lib.g5_bfs_validate_renumbered(_ptr(g.sr.rowstarts), _ptr(g.sr.col), g.nglobalverts, root, _ptr(pred),
                                              _ptr(dist), _ptr(g.sr.perm), _ptr(g.sr.inv), _ptr(work), work.numel(),
                                              C.byref(out), _stream(stream)))
    else:
        _check(lib.g5_bfs_validate(_ptr(g.rowstarts), _ptr(g.col), g.nglobalverts, root, _ptr(pred), _ptr(dist),
                                   _ptr(work), work.numel(), C.byref(out), _stream(stream)))
    return out.value


def sssp_validate(g: OnedGraph, root: int, dist: torch.Tensor, pred: torch.Tensor,
                  work: torch.Tensor | None = None, stream=None) -> int:
    """Error count of the SSSP rules (no counterpart in the reference); on the
    SSSP's renumbered copy when the graph has one (the same count)."""
    work = _val_work(g) if work is None else work
    out = C.c_uint64()
    if g.sr is not None:
        _check(lib.g5_sssp_validate_renumbered(_ptr(g.sr.rowstarts), _ptr(g.sr.col), _ptr(g.sr.w), g.nglobalverts,
                                               root, _ptr(dist), _ptr(pred), _ptr(g.sr.perm), _ptr(g.sr.inv),
                                               _ptr(work), work.numel(), C.byref(out), _stream(stream)))
    else:
        _check(lib.g5_sssp_validate(_ptr(g.rowstarts), _ptr(g.col), _ptr(g.w), g.nglobalverts, root, _ptr(dist),
                                    _ptr(pred), _ptr(work), work.numel(), C.byref(out), _stream(stream)))
    return out.value
