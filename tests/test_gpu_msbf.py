"""Tiled form of stage 1's SSSP (multi-source Bellman-Ford over in-edges,
128 sources per tile) against the frontier form and the reference on every
golden fixture: int32 bit-exact, float32 within 1e-5 relative with
reachability exact; the round bound still reports FAP_ERR_NOT_CONVERGED."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from fastapsp_b200 import FAP_DTYPE_F32, FAP_MODE_BATCHED, Context, DeviceGraph, FapError
from fastapsp_b200 import _lib as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dg(case):
    ctx = Context(0)
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
    dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"],
                 case["bdy_num"])
    dg.set_param("stage1", 1)      # the SSSP form of stage 1
    return ctx, dg


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
def test_tiled_sssp_matches_frontier_and_reference(cuda_ok, name):
    case = load_golden(name)
    K, integral = int(case["K"]), bool(case["integral"])
    ctx, dg = _dg(case)
    dg.set_param("sssp_form", 1)
    dg.solve(mode=FAP_MODE_BATCHED)
    ref = _blocks(dg, K)
    dg.set_param("sssp_form", 2)
    dg.solve(mode=FAP_MODE_BATCHED)
    got = _blocks(dg, K)
    _close(got, ref, integral)
    if "dist" in case:
        _close(got, case["dist"], integral)
    else:
        np.testing.assert_array_equal(O.row_checksums(O.to_i32(got)), case["row_checksums"])
    # the resident cache built with the tiled form
    dg.cache_build()
    dg.solve(mode=FAP_MODE_BATCHED)
    _close(_blocks(dg, K), got, True)


def test_tiled_sssp_round_bound(cuda_ok):
    case = load_golden("grid64_k8")
    ctx, dg = _dg(case)
    dg.set_param("sssp_form", 2)
    dg.set_param("sssp_max_rounds", 3)
    with pytest.raises(FapError) as e:
        dg.solve(mode=FAP_MODE_BATCHED)
    assert e.value.code == L.FAP_ERR_NOT_CONVERGED
    dg.set_param("sssp_max_rounds", 0)
    dg.solve(mode=FAP_MODE_BATCHED)
    cs = np.concatenate([dg.block_checksums(p) for p in range(1, int(case["K"]) + 1)])
    np.testing.assert_array_equal(cs, case["row_checksums"])


@pytest.mark.parametrize("name", ["grid64_k8", "rmat8_f32_k4", "rmat8_int_k4"])
@pytest.mark.parametrize("form", ["sssp", "bgraph"])
def test_tiles_side_by_side_or_one_at_a_time(cuda_ok, name, form):
    """The same blocks whether the 128-source tiles run side by side (the
    default memory budget) or one at a time (tile_mb = 0.1, smaller than
    one tile: every tile its own group, the stamps carried from group to
    group), in the tiled SSSP form and in the Bellman-Ford closure of the
    boundary graph."""
    case = load_golden(name)
    K, integral = int(case["K"]), bool(case["integral"])
    if form == "bgraph" and not integral:
        pytest.skip("the boundary-graph form is compared bit for bit on int32 graphs")
    ctx, dg = _dg(case)
    if form == "sssp":
        dg.set_param("sssp_form", 2)
    else:
        dg.set_param("stage1", 2)
        dg.set_param("bgraph_form", 2)
    outs = []
    for mb in (96, 0.1):
        dg.set_param("tile_mb", mb)
        dg.solve(mode=FAP_MODE_BATCHED)
        dg.check()
        outs.append(_blocks(dg, K))
    _close(outs[1], outs[0], True)
    if "dist" in case:
        _close(outs[0], case["dist"], integral)
