"""The reference's edge-list dump format through the compat API
(tuple_graph_dump / tuple_graph_load, src/graph_generation.cu:314-396): a
graph dumped in two ranges at their offsets loads back byte for byte, whole
and as a sub-range at an odd offset, and builds the same CSR -- at SCALE 12
and at a size whose edge file exceeds 2 GiB (where the reference's int byte
counts overflow; this implementation counts in 64 bits)."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

from tests.conftest import PKG_DIR, REPO

pytestmark = pytest.mark.gpu

SRC = os.path.join(REPO, "tests", "compat_dump_load.cu")
LIB = os.path.join(PKG_DIR, "lib", "libg500b.a")


@pytest.fixture(scope="module")
def prog(tmp_path_factory):
    if not os.path.exists(LIB):
        pytest.skip("lib/libg500b.a not built")
    out = tmp_path_factory.mktemp("dumpload") / "compat_dump_load"
    cmd = ["/usr/local/cuda/bin/nvcc", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(REPO, "include", "compat"), "-I", os.path.join(REPO, "include", "compat", "shim"),
           "-o", str(out), SRC, LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return str(out)


def _run(prog, cwd, scale, ef):
    r = subprocess.run([prog, str(scale), str(ef)], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.startswith("ok"), (r.stdout[-1000:], r.stderr[-1000:])
    _, m, nbytes = r.stdout.split()
    assert int(m) == ef << scale
    assert os.path.getsize(os.path.join(cwd, "graph-refactor.bin")) == int(nbytes)
    assert os.path.getsize(os.path.join(cwd, "graph-refactor.bin.weights")) == 4 * int(m)
    return int(nbytes)


def test_dump_load_round_trip_scale12(prog, tmp_path):
    _run(prog, tmp_path, 12, 16)


def test_dump_load_round_trip_above_2gib(prog, tmp_path):
    # SCALE 23, edgefactor 18: 151M edges, a 2.4 GB edge file (+0.6 GB weights).
    if shutil.disk_usage(tmp_path).free < 8 << 30:
        pytest.skip("less than 8 GiB of free disk for the 3 GB dump")
    assert _run(prog, tmp_path, 23, 18) > 2 << 30
