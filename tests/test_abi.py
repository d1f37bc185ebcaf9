"""The C ABI library loads, exports every function include/g500b.h declares,
and its host-side functions match the reference's (golden fixtures).  No
device work: these run without a GPU."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

from tests.conftest import REPO


def header_functions():
    text = open(os.path.join(REPO, "include", "g500b.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char \*)\s*(g5_\w+)\(", text, re.M)))


def test_exports_every_declared_symbol(cgt):
    names = header_functions()
    assert len(names) >= 20
    lib = C.CDLL(cgt.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_function(cgt):
    """Every declared function has a ctypes signature in the Python mirror
    (an unbound one would pass 64-bit pointers and sizes as C ints).
    g5_bfs_run_static is bound by its own test."""
    unbound = [n for n in header_functions() if n != "g5_bfs_run_static" and getattr(cgt.lib, n).argtypes is None]
    assert not unbound, unbound


def test_host_functions_match_reference(cgt, golden_host):
    for k in golden_host["make_mrg_seed"]:
        assert cgt.make_mrg_seed(k["s1"], k["s2"]) == k["seed"]
    for k in golden_host["make_random_numbers"]:
        got = cgt.make_random_numbers(8, k["s1"], k["s2"], k["position"])
        assert [float(x).hex() for x in got] == k["values_hex"]
    for k in golden_host["scramble_keys"]:
        assert cgt.scramble_keys(cgt.make_mrg_seed(k["s1"], k["s2"])) == (k["val0"], k["val1"])


def test_argument_errors_need_no_device(cgt):
    lib = cgt.lib
    seed = (C.c_uint32 * 5)(3, 1, 4, 1, 1)
    assert lib.g5_generate_kronecker_range(seed, 0, 0, 10, None, None, None) == -1
    assert b"log_n" in lib.g5_last_error()
    bad = (C.c_uint32 * 5)(0x7FFFFFFF, 1, 1, 1, 1)
    assert lib.g5_generate_kronecker_range(bad, 12, 0, 10, None, None, None) == -1
    zero = (C.c_uint32 * 5)(0, 0, 0, 0, 0)
    assert lib.g5_generate_kronecker_range(zero, 12, 0, 10, None, None, None) == -1
    # empty range: nothing to do, no pointer needed
    assert lib.g5_generate_kronecker_range(seed, 12, 5, 5, None, None, None) == 0
    assert lib.g5_bfs_run(None, None, 16, 16, None, None, None, 0, None, None) == -1
    assert b"root" in lib.g5_last_error()
    assert lib.g5_sssp_run(None, None, None, None, 0.1, 16, 99, None, None, None, 0, None, None) == -1
    assert lib.g5_csr_count(None, 0, 0, None, None, 0, None, None) == -1
    nb = C.c_uint64()
    assert lib.g5_msbfs_workspace_size(1 << 10, 1 << 14, 9, C.byref(nb)) == -1
    assert lib.g5_msbfs_workspace_size(1 << 10, 1 << 14, 0, C.byref(nb)) == 0 and nb.value > 0
    roots = (C.c_uint64 * 2)(1, 2)
    assert lib.g5_msbfs_run(16, 100, 0, roots, 2, None, 0, None, None, None) == -1
    assert lib.g5_msbfs_prepare(None, None, 0, 0, 0, None, 0, None) == -1


def test_workspace_sizes_scale_with_vertices(cgt):
    for fn in ("g5_bfs_workspace_size", "g5_sssp_workspace_size", "g5_validate_workspace_size"):
        small, big = C.c_uint64(), C.c_uint64()
        assert getattr(cgt.lib, fn)(1 << 10, C.byref(small)) == 0
        assert getattr(cgt.lib, fn)(1 << 20, C.byref(big)) == 0
        assert big.value > small.value > 0
    b = C.c_uint64()
    assert cgt.lib.g5_csr_workspace_size(1 << 20, 16 << 20, C.byref(b)) == 0 and b.value > 4 << 20
