"""Drop-in check: the reference's examples/graph500_runner.cu, compiled
unchanged against include/compat (+ the single-process MPI/NVSHMEM shims)
and linked with libg500b, builds and runs: 64 validated BFS roots, SSSP, the
edge-list dump in the reference's file format, and the TEPS edge counts of
the reference's own run (golden fixtures)."""
from __future__ import annotations

import hashlib
import os
import re
import subprocess

import numpy as np
import pytest

from tests.conftest import PKG_DIR, REPO, load_golden



def _ref_root() -> str:
    """The reference checkout: G5_REF_ROOT, else the one the build used
    (recorded by __graft_entry__.build in oracle/_ref/REF_ROOT)."""
    root = os.environ.get("G5_REF_ROOT", "")
    rec = os.path.join(REPO, "oracle", "_ref", "REF_ROOT")
    if not root and os.path.exists(rec):
        root = open(rec).read().strip()
    return root


REF_RUNNER_SRC = os.path.join(_ref_root(), "examples", "graph500_runner.cu") if _ref_root() else ""
RUNNER = os.path.join(PKG_DIR, "lib", "graph500_runner")


@pytest.mark.skipif(not REF_RUNNER_SRC or not os.path.exists(REF_RUNNER_SRC),
                    reason="reference sources not present on this machine")
def test_runner_compiles_unchanged(tmp_path):
    out = tmp_path / "runner"
    cmd = ["/usr/local/cuda/bin/nvcc", "-O1", "-Drestrict=__restrict__",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(REPO, "include", "compat"), "-I", os.path.join(REPO, "include", "compat", "shim"),
           "-c", "-o", str(out) + ".o", REF_RUNNER_SRC]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


def _stats(text: str) -> dict[str, float]:
    out = {}
    for line in text.splitlines():
        m = re.match(r"^(.*?):\s+!?\s*([-+0-9.eE]+)\s*$", line)
        if m:
            out[m.group(1).strip()] = float(m.group(2))
    return out


@pytest.mark.gpu
def test_runner_scale12_matches_reference(tmp_path):
    if not os.path.exists(RUNNER):
        pytest.skip("runner not built (make -C cuda-graph-traversal_b200 runner)")
    r = subprocess.run([RUNNER, "12", "16"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Validation failed" not in r.stderr
    s = _stats(r.stdout)
    fx = load_golden("ref_s12.json")
    nedges = np.array([p["nedge"] for p in fx["per_root"]], np.float64)
    assert s["SCALE"] == 12 and s["edgefactor"] == 16 and s["NBFS"] == 64
    assert s["min_nedge"] == nedges.min() and s["max_nedge"] == nedges.max()
    assert s["mean_nedge"] == pytest.approx(nedges.mean(), rel=1e-12)
    assert s["bfs  harmonic_mean_TEPS"] > 0 and s["sssp median_TEPS"] > 0
    # tuple_graph_dump wrote the reference's raw format.
    edges = np.fromfile(tmp_path / "graph-refactor.bin", np.uint64)
    weights = np.fromfile(tmp_path / "graph-refactor.bin.weights", np.float32)
    assert hashlib.sha256(edges.tobytes()).hexdigest() == fx["edges_sha256"]
    assert hashlib.sha256(weights.tobytes()).hexdigest() == fx["weights_sha256"]


@pytest.mark.gpu
def test_runner_skip_flags_and_dot(tmp_path):
    if not os.path.exists(RUNNER):
        pytest.skip("runner not built")
    env = dict(os.environ, SKIP_SSSP="1", SKIP_VALIDATION="1", WRITE_DOT="1")
    r = subprocess.run([RUNNER, "6", "4"], cwd=tmp_path, capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "sssp" not in r.stdout and "validate" not in r.stdout
    names = set(os.listdir(tmp_path / "dot"))
    assert {"tuple_pe_000.dot", "tuple_global.dot", "oned_pe_000.dot", "oned_global.dot",
            "bfs_000_pe_000.dot", "bfs_000_global.dot"} <= names
    text = (tmp_path / "dot" / "bfs_000_global.dot").read_text()
    assert text.startswith("digraph bfs_global {") and "pred" in text
    bad = subprocess.run([RUNNER], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert bad.returncode != 0 and "Usage" in bad.stderr
