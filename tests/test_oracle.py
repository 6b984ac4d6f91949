"""The oracle (C restatement of the reference's CPU path) against the
reference's own outputs: the committed golden fixtures everywhere, and the
reference binary itself when it is built here (oracle/_ref)."""
import os
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden_names, load_golden
from oracle import oracle as O


def meta_of(case):
    return O.Meta(case["n"], case["m"], case["K"], case["row_offset"], case["col_val"],
                  case["weight"], case["graph_id"], case["st2ed"],
                  np.argsort(case["st2ed"]).astype(np.int32), case["ver_num"],
                  case["ver_offset"], case["bdy_num"])


def _solve_port(case):
    out = O.port_solve_meta(meta_of(case))
    return np.concatenate([out[p] for p in range(1, case["K"] + 1)], 0)


@pytest.mark.parametrize("name", golden_names())
def test_port_matches_reference_fixture(name):
    case = load_golden(name)
    full = _solve_port(case)
    if "dist" in case:
        if case["integral"]:
            assert np.array_equal(full.view(np.int32), case["dist"].view(np.int32))
        else:
            ref = case["dist"]
            reach = ref < 1e8
            assert np.array_equal(reach, full < 1e8)
            rel = np.abs(full[reach] - ref[reach]) / np.maximum(np.abs(ref[reach]), 1e-30)
            assert rel.max(initial=0) <= 1e-5
    else:
        cs = O.row_checksums(O.to_i32(full))
        assert np.array_equal(cs, case["row_checksums"])
        assert np.array_equal(full[case["sample_rows"]], case["sample_dist"])


@pytest.mark.parametrize("name", golden_names())
def test_fixture_partition_contract(name):
    """st2ed / counts obey the sort_and_encode contract for the fixture's
    partition (restated in numpy from util_preprocess.h:32-106)."""
    c = load_golden(name)
    flag = O.restate_boundary(c["row_offset"], c["col_val"], c["graph_id"])
    O.check_encoding(c["st2ed"], c["graph_id"], flag, c["K"])
    vn, vo, bn = O.restate_encode_classes(c["graph_id"], flag, c["K"])
    assert np.array_equal(vn[1:], c["ver_num"][1:])
    assert np.array_equal(vo[1:], c["ver_offset"][1:])
    assert np.array_equal(bn[1:], c["bdy_num"][1:])


@pytest.mark.parametrize("name", ["grid12_k4", "road300_k6", "disconnected_k3", "rmat8_int_k4"])
def test_fixture_against_scipy(name):
    """Independent check: where inner rows have no duplicate-edge quirk, the
    reference's distances are the true shortest paths."""
    sp = pytest.importorskip("scipy.sparse.csgraph")
    from scipy.sparse import csr_matrix
    c = load_golden(name)
    n = c["n"]
    ro, col, w = c["row_offset"], c["col_val"], c["weight"]
    # scipy keeps the minimum of duplicate entries
    src = np.repeat(np.arange(n), np.diff(ro))
    best = {}
    for a, b, x in zip(src.tolist(), col.tolist(), w.tolist()):
        if a == b:
            continue
        if (a, b) not in best or x < best[(a, b)]:
            best[(a, b)] = x
    rows = np.array([k[0] for k in best]), np.array([k[1] for k in best])
    M = csr_matrix((np.array(list(best.values())), rows), shape=(n, n))
    D = sp.shortest_path(M, directed=True, method="D")
    D[np.isinf(D)] = 1e8
    ref = c["dist"].astype(np.float64)
    truth = D[c["st2ed"]]
    # the reference's inner rows use the last duplicate edge, which can only
    # lengthen paths; every entry is >= the true distance and boundary rows
    # are exact
    assert np.all(ref >= truth - 1e-3)
    start = c["ver_offset"]
    for p in range(1, c["K"] + 1):
        b = c["bdy_num"][p]
        np.testing.assert_array_equal(ref[start[p]:start[p] + b], truth[start[p]:start[p] + b])
    if name != "road300_k6" and name != "rmat8_int_k4":
        np.testing.assert_array_equal(ref, truth)


def test_dijkstra_port_simple():
    # 0 -> 1 (5), 0 -> 2 (1), 2 -> 1 (1), 3 isolated
    ro = np.array([0, 2, 2, 3, 3], np.int32)
    col = np.array([1, 2, 1], np.int32)
    w = np.array([5, 1, 1], np.float32)
    d = O.port_dijkstra(ro, col, w, 0)
    assert d.tolist() == [0.0, 2.0, 1.0, 1e8]


@pytest.mark.skipif(not O.ref_available(), reason="reference binary not built here")
@pytest.mark.parametrize("seed", [21, 22])
def test_port_matches_reference_binary(seed):
    """Fresh random graphs: the restatement and the reference agree bit for bit."""
    from fastapsp_b200 import generators as G
    g = G.road_graph(400, seed=seed, wmin=1, wmax=50)
    with tempfile.TemporaryDirectory() as tmp:
        G.write_mtx(g, tmp, "r")
        meta_f = os.path.join(tmp, "m.bin")
        dist_f = os.path.join(tmp, "d.bin")
        O.run_ref(tmp, "r", False, True, 5, meta_out=meta_f, dist_out=dist_f)
        meta = O.read_meta(meta_f)
        ref = np.fromfile(dist_f, np.float32).reshape(meta.n, meta.n)
    out = O.port_solve_meta(meta)
    full = np.concatenate([out[p] for p in range(1, meta.K + 1)], 0)
    assert np.array_equal(full.view(np.int32), ref.view(np.int32))


@pytest.mark.skipif(not O.ref_available(), reason="reference binary not built here")
def test_reference_row_checksums_and_shared_partition():
    """fap_ref --rowsum writes the per-row checksums of its int32-cast blocks
    (the same formula as the library's fap_graph_block_checksums), and a
    partition given through FAP_PARTITION_FILE replaces its METIS call; a
    checksum changed on the oracle side is caught by the bench's comparison."""
    import importlib.util
    from fastapsp_b200 import generators as G
    g = G.road_graph(500, seed=3, wmin=1, wmax=100)
    K = 5
    with tempfile.TemporaryDirectory() as tmp:
        G.write_mtx(g, tmp, "r")
        meta_f = os.path.join(tmp, "m.bin")
        dist_f = os.path.join(tmp, "d.bin")
        sum_f = os.path.join(tmp, "s.bin")
        part_f = os.path.join(tmp, "p.bin")
        gid0 = (np.arange(g.n) * K // g.n).astype(np.int32)
        gid0.tofile(part_f)
        O.run_ref(tmp, "r", False, True, K, parts=[2, 4], meta_out=meta_f, dist_out=dist_f,
                  rowsum_out=sum_f, partition_file=part_f)
        meta = O.read_meta(meta_f)
        assert np.array_equal(meta.graph_id, gid0 + 1)
        dist = np.fromfile(dist_f, np.float32).reshape(-1, meta.n)
        sums = np.fromfile(sum_f, np.uint64)
        assert np.array_equal(sums, O.row_checksums(O.to_i32(dist)))
        # the bench's comparison: equal sums pass, one planted change is a mismatch
        spec = importlib.util.spec_from_file_location(
            "bench_parity", os.path.join(ROOT, "bench.py"))
        b = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(b)
        s2 = int(meta.ver_num[2])
        gpu = {2: sums[:s2].copy(), 4: sums[s2:].copy()}
        f2, f4 = os.path.join(tmp, "s2.bin"), os.path.join(tmp, "s4.bin")
        sums[:s2].tofile(f2)
        planted = sums[s2:].copy()
        planted[3] += np.uint64(1)
        planted.tofile(f4)

        class W:
            name, n = "r", meta.n
        res = b.compare_parity(W, gpu, {2: f2, 4: f4}, 0, meta.st2ed, meta)
        assert res["parts"] == 2 and res["rows"] == sums.size and res["mismatches"] == 1
        assert res["st2ed_equal"] is True


def _path_names():
    return [n for n in golden_names() if "path" in load_golden(n)]


def _duplicate_free(case):
    ro, col = case["row_offset"], case["col_val"]
    for u in range(int(case["n"])):
        nb = col[ro[u]:ro[u + 1]].tolist()
        if len(set(nb)) != len(nb) or u in nb:
            return False
    return True


@pytest.mark.parametrize("name", _path_names())
def test_predecessor_rule_matches_reference_paths(name):
    """The predecessor rule of the B200 path (argmin over in-edges, smallest
    vertex on ties), applied to the reference's distances, gives the
    reference's own predecessor matrix on every entry whose predecessor is
    unique (there every evaluation order must agree)."""
    c = load_golden(name)
    rows = c["st2ed"]
    integral = bool(c["integral"])
    P = O.port_predecessors(c["dist"], rows, c["row_offset"], c["col_val"], c["weight"], integral)
    U = O.unique_predecessor_mask(c["dist"], rows, c["row_offset"], c["col_val"], c["weight"], integral)
    assert U.sum() > 0
    np.testing.assert_array_equal(P[U], c["path"][U])
    # sources and unreachable entries agree everywhere
    n = int(c["n"])
    np.testing.assert_array_equal(P[np.arange(n), rows], c["path"][np.arange(n), rows])
    unreach = c["dist"] >= 1e8
    np.testing.assert_array_equal(P[unreach], c["path"][unreach])


@pytest.mark.parametrize("name", [n for n in _path_names() if _duplicate_free(load_golden(n))])
def test_reference_and_rule_paths_are_valid(name):
    """On graphs without duplicate edges or self-loops (where the reference's
    in-part distances are true shortest distances), both the reference's
    predecessor matrix and the rule's pass the validity check."""
    c = load_golden(name)
    args = (c["st2ed"], c["row_offset"], c["col_val"], c["weight"], bool(c["integral"]))
    assert O.check_paths(c["dist"], c["path"], *args) > 0
    P = O.port_predecessors(c["dist"], *args)
    assert O.check_paths(c["dist"], P, *args) > 0


def test_check_paths_catches_a_planted_error():
    c = load_golden("grid12_k4")
    args = (c["st2ed"], c["row_offset"], c["col_val"], c["weight"], True)
    P = c["path"].copy()
    r, j = 5, int(np.nonzero(c["dist"][5] > 3)[0][0])
    P[r, j] = c["st2ed"][r]          # the source is not adjacent to j
    with pytest.raises(AssertionError):
        O.check_paths(c["dist"], P, *args)


@pytest.mark.parametrize("name", _path_names())
def test_min_plus_predecessor_rule_matches_reference_paths(name):
    """The rule the GPU uses for inner rows of parts with few boundary
    vertices (the predecessor on the row of the boundary vertex the min-plus
    merge chose), applied to the reference's distances: equal to the
    reference's predecessors wherever unique, valid everywhere (graphs
    without duplicate arcs)."""
    c = load_golden(name)
    integral = bool(c["integral"])
    args = (c["row_offset"], c["col_val"], c["weight"], integral)
    P = O.port_predecessors_parts(c["dist"], c["st2ed"], c["ver_num"], c["ver_offset"], c["bdy_num"], *args)
    U = O.unique_predecessor_mask(c["dist"], c["st2ed"], *args)
    np.testing.assert_array_equal(P[U], c["path"][U])
    if _duplicate_free(c):
        assert O.check_paths(c["dist"], P, c["st2ed"], *args) > 0
