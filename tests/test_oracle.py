"""The CPU oracle against the reference's own outputs (golden fixtures made
by tests/golden/make_golden.py from the reference built by oracle/ref.mk),
plus the oracle's internal consistency.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from tests.golden.make_golden import canonical_csr, golden_hashes, sha


def test_make_mrg_seed(oracle, golden_host):
    for k in golden_host["make_mrg_seed"]:
        assert oracle.make_mrg_seed(k["s1"], k["s2"]).tolist() == k["seed"]


def test_make_random_numbers(oracle, golden_host):
    for k in golden_host["make_random_numbers"]:
        got = oracle.make_random_numbers(8, k["s1"], k["s2"], k["position"])
        assert [float(x).hex() for x in got] == k["values_hex"]


def test_mrg_jump_matches_reference_table(oracle, golden_host):
    """The oracle recomputes the reference's byte-indexed jump table; 96
    random jumps over all 24 byte positions agree with the reference's."""
    L = oracle.lib()
    import ctypes as C
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    L.orc_mrg_skip.argtypes = [u32p, C.c_uint64, C.c_uint64, C.c_uint64]
    for k in golden_host["mrg_skip"]:
        z = np.array(k["state"], np.uint32)
        L.orc_mrg_skip(z, k["high"], k["mid"], k["low"])
        assert z.tolist() == k["result"]


def test_mrg_draws(oracle, golden_host):
    import ctypes as C
    L = oracle.lib()
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    L.orc_mrg_draw.argtypes = [u32p, C.c_int, u32p]
    z = np.array([3, 1, 4, 1, 1], np.uint32)
    out = np.zeros(64, np.uint32)
    L.orc_mrg_draw(z, 64, out)
    assert out.tolist() == golden_host["mrg_draws_from_seed_2_3"]


def test_scramble_keys(oracle, golden_host):
    for k in golden_host["scramble_keys"]:
        assert oracle.scramble_keys(oracle.make_mrg_seed(k["s1"], k["s2"])) == (k["val0"], k["val1"])


@pytest.fixture(scope="module")
def oracle_graphs(oracle):
    out = {}
    for scale in (12, 14):
        seed = oracle.make_mrg_seed(2, 3)
        e, w = oracle.generate_kronecker_range(seed, scale, 0, 16 << scale)
        rs, col, cw = oracle.csr_build(e, w, 1 << scale)
        out[scale] = (e, w, rs, col, cw)
    return out


def test_generator_and_csr_match_reference(oracle_graphs, golden_dump):
    e, w, rs, col, cw = oracle_graphs[golden_dump["scale"]]
    assert e.shape[0] == golden_dump["nedges"]
    assert e[:16].tolist() == golden_dump["first_edges"]
    assert [float(x).hex() for x in w[:16]] == golden_dump["first_weights_hex"]
    h = golden_hashes(e, w, rs, col, cw)
    for k, v in h.items():
        assert v == golden_dump[k], k
    assert int(rs[-1]) == golden_dump["nentries"]
    assert int((e[:, 0] == e[:, 1]).sum()) == golden_dump["self_loops"]
    assert int((np.diff(rs.astype(np.int64)) == 0).sum()) == golden_dump["isolated"]


def test_roots_match_reference(oracle, oracle_graphs, golden_dump):
    scale = golden_dump["scale"]
    rs = oracle_graphs[scale][2]
    roots = oracle.generate_bfs_roots(rs, 1 << scale, 2, 3, len(golden_dump["roots"]))
    assert roots.tolist() == golden_dump["roots"]


def test_bfs_sssp_match_reference(oracle, oracle_graphs, golden_dump):
    """Depth arrays (the reference's bfs_compute_dist_from_pred of its own
    BFS) and float32 SSSP distances (its delta-stepping) are bit-identical
    to the oracle's; nedge and reached counts agree."""
    scale = golden_dump["scale"]
    n = 1 << scale
    _, _, rs, col, cw = oracle_graphs[scale]
    for pr in golden_dump["per_root"]:
        r = pr["root"]
        pred, depth = oracle.bfs(rs, col, n, r)
        assert sha(depth) == pr["depth_sha256"], r
        assert oracle.edge_count(rs, col, n, pred) == pr["nedge"]
        assert int((pred != -1).sum()) == pr["reached"]
        dist, spred = oracle.sssp(rs, col, cw, n, r)
        assert sha(dist) == pr["sssp_dist_sha256"], r
        assert oracle.sssp_validate(rs, col, cw, n, r, dist, spred) == 0


def test_depth_fixture_array(oracle, oracle_graphs):
    data = np.load(__import__("os").path.join(__import__("tests.conftest", fromlist=["GOLDEN"]).GOLDEN,
                                              "ref_s12_depth.npz"))["depth"]
    from tests.conftest import load_golden
    fx = load_golden("ref_s12.json")
    _, _, rs, col, _ = oracle_graphs[12]
    for i, pr in enumerate(fx["per_root"][:8]):
        _, depth = oracle.bfs(rs, col, 4096, pr["root"])
        assert np.array_equal(depth.astype(np.int8), data[i])


def test_bfs_validator_and_dist_from_pred(oracle, oracle_graphs):
    _, _, rs, col, _ = oracle_graphs[12]
    n = 4096
    for r in oracle.generate_bfs_roots(rs, n, 2, 3, 8).tolist():
        pred, depth = oracle.bfs(rs, col, n, r)
        dist = oracle.bfs_dist_from_pred(rs, col, n, pred, r)
        assert np.array_equal(dist, depth)
        assert oracle.bfs_validate(rs, col, n, r, pred, dist) == 0


def test_planted_mistakes_are_caught(oracle, oracle_graphs):
    """Corrupted parent trees and depths (planted on the CPU) fail the
    runner's rules; unreachable parent chains leave INT64_MAX depths."""
    _, _, rs, col, cw = oracle_graphs[12]
    n = 4096
    r = int(oracle.generate_bfs_roots(rs, n, 2, 3, 1)[0])
    pred, depth = oracle.bfs(rs, col, n, r)
    reached = np.nonzero((pred != -1) & (np.arange(n) != r))[0]
    bad = pred.copy()
    bad[reached[:5]] = reached[10:15]          # parents that are (mostly) not neighbours
    dist = oracle.bfs_dist_from_pred(rs, col, n, bad, r)
    assert (dist == np.iinfo(np.int64).max).any()
    assert oracle.bfs_validate(rs, col, n, r, bad, dist) > 0
    out_of_range = pred.copy()
    out_of_range[reached[0]] = n + 7
    d2 = oracle.bfs_dist_from_pred(rs, col, n, out_of_range, r)
    assert oracle.bfs_validate(rs, col, n, r, out_of_range, d2) > 0
    skew = depth.copy()
    skew[reached[0]] += 2
    assert oracle.bfs_validate(rs, col, n, r, pred, skew) > 0
    sd, sp = oracle.sssp(rs, col, cw, n, r)
    sd2 = sd.copy()
    sd2[reached[3]] += np.float32(0.25)
    assert oracle.sssp_validate(rs, col, cw, n, r, sd2, sp) > 0
