"""Boundary-graph form of stage 1 (local closures + APSP over the boundary
vertices + expansion) against the SSSP form and the reference: int32
bit-exact, float32 within 1e-5 relative with reachability exact; batched,
cached, with predecessor rows, and the automatic choice (int32 graphs
without duplicate arcs inside a part; float32 only on request)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from fastapsp_b200 import FAP_DTYPE_F32, FAP_MODE_BATCHED, Context, DeviceGraph
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dg(case):
    ctx = Context(0)
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
    dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"],
                 case["bdy_num"])
    return ctx, dg


def _dup_inside_parts(case):
    ro, col, gid = case["row_offset"], case["col_val"], case["graph_id"]
    for u in range(int(case["n"])):
        nb = [int(v) for v in col[ro[u]:ro[u + 1]] if gid[v] == gid[u]]
        if len(set(nb)) != len(nb):
            return True
    return False


def _blocks(dg, K):
    return np.concatenate([dg.copy_block(p, out_dtype=FAP_DTYPE_F32) for p in range(1, K + 1)], 0)


def _close(a, b, integral):
    if integral:
        np.testing.assert_array_equal(a.view(np.int32), b.view(np.int32))
    else:
        reach = b < 1e8
        assert np.array_equal(reach, a < 1e8)
        rel = np.abs(a[reach] - b[reach]) / np.maximum(np.abs(b[reach]), 1e-30)
        assert rel.max(initial=0.0) <= 1e-5


@pytest.mark.parametrize("name", golden_names())
def test_boundary_graph_matches_sssp_and_reference(cuda_ok, name):
    case = load_golden(name)
    K, integral = int(case["K"]), bool(case["integral"])
    ctx, dg = _dg(case)
    dg.set_param("stage1", 1)
    dg.solve(mode=FAP_MODE_BATCHED)
    assert dg.last_stage1() == 1
    ref = _blocks(dg, K)
    dg.set_param("stage1", 0)
    dg.solve(mode=FAP_MODE_BATCHED)
    usable = not _dup_inside_parts(case) and int(case["bdy_num"][1:].sum()) > 0
    assert dg.last_stage1() == (2 if usable and integral else 1)
    if usable and not integral:   # float32: only on request (rounding order differs)
        dg.set_param("stage1", 2)
        dg.solve(mode=FAP_MODE_BATCHED)
        assert dg.last_stage1() == 2
    got = _blocks(dg, K)
    _close(got, ref, integral)
    if "dist" in case:
        _close(got, case["dist"], integral)
    else:
        np.testing.assert_array_equal(O.row_checksums(O.to_i32(got)), case["row_checksums"])
    # the resident cache built the same way
    dg.cache_build()
    dg.solve(mode=FAP_MODE_BATCHED)
    assert dg.last_stage1() == 3
    _close(_blocks(dg, K), got, True)
    src = list(range(0, int(case["n"]), max(1, int(case["n"]) // 40)))
    rows = dg.rows(src)
    ed2st = np.empty(int(case["n"]), np.int64)
    ed2st[case["st2ed"]] = np.arange(int(case["n"]))
    _close(rows, got[ed2st[src]], True)


@pytest.mark.parametrize("name", ["grid12_k4", "rgg300_f32_k4", "disconnected_k3"])
def test_boundary_graph_with_paths(cuda_ok, name):
    case = load_golden(name)
    K = int(case["K"])
    ctx, dg = _dg(case)
    dg.set_param("paths", 1)
    dg.set_param("stage1", 2)
    dg.solve(mode=FAP_MODE_BATCHED)
    assert dg.last_stage1() == 2
    D = _blocks(dg, K)
    P = np.concatenate([dg.copy_path_block(p) for p in range(1, K + 1)], 0)
    args = (case["st2ed"], case["row_offset"], case["col_val"], case["weight"], bool(case["integral"]))
    want = O.port_predecessors_parts(D, case["st2ed"], case["ver_num"], case["ver_offset"],
                                     case["bdy_num"], *args[1:])
    np.testing.assert_array_equal(P, want)
    assert O.check_paths(D, P, *args) > 0


@pytest.mark.parametrize("name", golden_names())
def test_bellman_ford_closure_and_tiled_expansion(cuda_ok, name):
    """bgraph_form 2: the boundary graph closed by the tiled Bellman-Ford over
    its in-edge CSR and the boundary rows written by the tiled expansion (the
    automatic choice above 8192 boundary vertices), forced on every fixture:
    the same blocks as the SSSP form and the reference, in one batch and
    from the resident cache."""
    case = load_golden(name)
    K, integral = int(case["K"]), bool(case["integral"])
    if _dup_inside_parts(case) or int(case["bdy_num"][1:].sum()) == 0:
        pytest.skip("boundary-graph form not applicable")
    ctx, dg = _dg(case)
    dg.set_param("stage1", 1)
    dg.solve(mode=FAP_MODE_BATCHED)
    ref = _blocks(dg, K)
    dg.set_param("stage1", 2)
    dg.set_param("bgraph_form", 2)
    dg.solve(mode=FAP_MODE_BATCHED)
    dg.check()
    assert dg.last_stage1() == 2
    got = _blocks(dg, K)
    _close(got, ref, integral)
    if "dist" in case:
        _close(got, case["dist"], integral)
    else:
        np.testing.assert_array_equal(O.row_checksums(O.to_i32(got)), case["row_checksums"])
    dg.solve(mode=FAP_MODE_BATCHED)    # again: local weights refreshed, CSR reused
    _close(_blocks(dg, K), got, True)
    dg.cache_build()
    dg.check()
    held, built = dg.cache_bytes()
    assert built and held > 0
    dg.solve(mode=FAP_MODE_BATCHED)
    assert dg.last_stage1() == 3
    assert dg.stage1_name() == "resident cache (boundary graph, Bellman-Ford closure)"
    _close(_blocks(dg, K), got, True)
    dg.cache_build(rebuild=True)     # stages 1-2 again in the same buffers
    dg.solve(mode=FAP_MODE_BATCHED)
    _close(_blocks(dg, K), got, True)
