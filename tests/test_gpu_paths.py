"""Predecessor (path) matrices on the GPU, through the C ABI.

For every golden fixture: the predecessor rows equal the rules' restatement
(oracle.port_predecessors_parts on the same distances) bit for bit, equal the
reference's own predecessor matrix wherever the predecessor is unique, and
pass the validity check (edge, distance equation, chain back to the source)
on graphs without duplicate edges; the same in the plain form, the batched
form with the one-CTA-per-part Floyd, and from the resident cache.  Then the
drop-in fapGraph getters and point-to-point paths.
"""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_names, load_golden, write_golden_mtx
from fastapsp_b200 import (FAP_DTYPE_F32, FAP_MODE_BATCHED, FAP_MODE_PLAIN, Context, DeviceGraph,
                           FapError, fapGraph)
from fastapsp_b200 import _lib as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PATH_CASES = [n for n in golden_names() if "path" in load_golden(n)]


def _dg(case):
    ctx = Context(0)
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
    dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"],
                 case["bdy_num"])
    return ctx, dg


def _all_rows(dg, K):
    D = np.concatenate([dg.copy_block(p, out_dtype=FAP_DTYPE_F32) for p in range(1, K + 1)], 0)
    P = np.concatenate([dg.copy_path_block(p) for p in range(1, K + 1)], 0)
    return D, P


def _duplicate_free(case):
    ro, col = case["row_offset"], case["col_val"]
    for u in range(int(case["n"])):
        nb = col[ro[u]:ro[u + 1]].tolist()
        if len(set(nb)) != len(nb) or u in nb:
            return False
    return True


def _check_case(case, D, P):
    integral = bool(case["integral"])
    args = (case["st2ed"], case["row_offset"], case["col_val"], case["weight"], integral)
    # the rules, restated on the CPU over the same distances: bit-exact
    want = O.port_predecessors_parts(D, case["st2ed"], case["ver_num"], case["ver_offset"],
                                     case["bdy_num"], case["row_offset"], case["col_val"],
                                     case["weight"], integral)
    np.testing.assert_array_equal(P, want)
    # the reference's own predecessors wherever the predecessor is unique
    U = O.unique_predecessor_mask(case["dist"], *args)
    np.testing.assert_array_equal(P[U], case["path"][U])
    if _duplicate_free(case):
        assert O.check_paths(D, P, *args) > 0


@pytest.mark.parametrize("form", ["batched", "plain", "per_cta", "cached"])
@pytest.mark.parametrize("name", PATH_CASES)
def test_paths_match_rule_and_reference(cuda_ok, name, form):
    case = load_golden(name)
    K = int(case["K"])
    ctx, dg = _dg(case)
    dg.set_param("paths", 1)
    if form == "per_cta":
        dg.set_param("floyd_per_cta", 1)
    if form == "cached":
        dg.cache_build()
    dg.solve(mode=FAP_MODE_PLAIN if form == "plain" else FAP_MODE_BATCHED)
    D, P = _all_rows(dg, K)
    _check_case(case, D, P)


def test_paths_on_grid64_sample_rows(cuda_ok):
    case = load_golden("grid64_k8")
    K = int(case["K"])
    ctx, dg = _dg(case)
    dg.set_param("paths", 1)
    dg.solve(mode=FAP_MODE_BATCHED)
    D, P = _all_rows(dg, K)
    # every part has more boundary vertices than the min-plus rule's limit, so
    # every row follows the in-edge rule
    assert int(case["bdy_num"][1:].min()) > O.PRED_THIN_B
    rows = np.sort(np.random.default_rng(4).choice(int(case["n"]), 48, replace=False))
    args = (case["st2ed"][rows], case["row_offset"], case["col_val"], case["weight"], True)
    np.testing.assert_array_equal(P[rows], O.port_predecessors(D[rows], *args))
    assert O.check_paths(D[rows], P[rows], *args) > 0


def test_paths_need_positive_weights(cuda_ok):
    # 0 -> 1 (w 0), 1 -> 2 (w 3), 2 -> 0 (w 1)
    ctx = Context(0)
    ro = np.array([0, 1, 2, 3], np.int32)
    col = np.array([1, 2, 0], np.int32)
    dg = DeviceGraph(ctx, ro, col, np.array([0, 3, 1], np.float32))
    with pytest.raises(FapError) as e:
        dg.set_param("paths", 1)
    assert e.value.code == L.FAP_ERR_RANGE


def test_block_without_paths_is_refused(cuda_ok):
    case = load_golden("grid12_k4")
    ctx, dg = _dg(case)
    dg.solve(mode=FAP_MODE_BATCHED)
    with pytest.raises(FapError) as e:
        dg.copy_path_block(1)
    assert e.value.code == L.FAP_ERR_STATE


@pytest.mark.parametrize("name", ["grid12_k4", "rgg300_f32_k4"])
def test_fapgraph_path_getters(cuda_ok, name):
    case = load_golden(name)
    n = int(case["n"])
    with tempfile.TemporaryDirectory() as tmp:
        write_golden_mtx(case, tmp)
        g = fapGraph(case["name"], bool(case["directed"]), bool(case["weighted"]), int(case["K"]),
                     root=tmp)
        if case["injected_partition"]:
            gid0 = (np.arange(n, dtype=np.int64) * case["K"] // n).astype(np.int32)
            g.setPartition(gid0 + 1)
        g.preCondition()
        assert g.solve(is_path_needed=True) == 0
        D, P = g.getAllDistance(), g.getAllPath()
        _check_case(case, D, P)
        # one part with paths: the same rows
        p = 2
        g.solveSubGraph(p, is_path_needed=True)
        off, rows = int(case["ver_offset"][p]), int(case["ver_num"][p])
        np.testing.assert_array_equal(g.getSubGraphPath(p), P[off:off + rows])
        v = int(case["st2ed"][off + 1])
        np.testing.assert_array_equal(g.getPathFromOnePoint(v), P[off + 1])
        # point-to-point paths: edges of the graph whose weights sum to the distance
        ro, col, w = case["row_offset"], case["col_val"], case["weight"]
        rng = np.random.default_rng(9)
        for _ in range(20):
            a, b = (int(x) for x in rng.integers(0, n, 2))
            path = g.getPathP2P(a, b)
            d = g.getDistanceP2P(a, b)
            if d >= 1e8:
                assert path == []
                continue
            assert path[0] == a and path[-1] == b
            total = 0.0
            for x, y in zip(path[:-1], path[1:]):
                ws = [float(w[e]) for e in range(ro[x], ro[x + 1]) if col[e] == y]
                assert ws, f"{x} -> {y} is not an edge"
                total += min(ws)
            assert abs(total - d) <= (0 if case["integral"] else 1e-4 * max(d, 1.0))


@pytest.mark.parametrize("name", ["grid12_k4", "rgg300_f32_k4"])
def test_fapgraph_paths_with_bounded_resident_rows(cuda_ok, name):
    """With fewer output rows allowed on the device than the graph has, the
    parts solved in groups (from the resident cache) give the same
    predecessor rows as one solve of every part."""
    case = load_golden(name)
    n, K = int(case["n"]), int(case["K"])
    with tempfile.TemporaryDirectory() as tmp:
        write_golden_mtx(case, tmp)
        g = fapGraph(case["name"], bool(case["directed"]), bool(case["weighted"]), K, root=tmp)
        if case["injected_partition"]:
            gid0 = (np.arange(n, dtype=np.int64) * K // n).astype(np.int32)
            g.setPartition(gid0 + 1)
        g.preCondition()
        assert g.solve(is_path_needed=True) == 0
        D, P = g.getAllDistance(), g.getAllPath()
        g.setMaxResidentRows(int(max(case["ver_num"][1:])))
        for p in range(K, 0, -1):
            g.solveSubGraph(p, is_path_needed=True)
            off, rows = int(case["ver_offset"][p]), int(case["ver_num"][p])
            np.testing.assert_array_equal(g.getSubGraphPath(p), P[off:off + rows])
            np.testing.assert_array_equal(g.getSubGraphDistance(p), D[off:off + rows])
