"""Resident cache (fap_graph_cache_build): batched solves and distance rows
served from the cached boundary rows and closed Floyd matrices give exactly
the values of the uncached path (bit-identical for int32 and float32: the
same min over the same sums), on every golden fixture, for both batched
Floyd forms, full and packed placements."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from fastapsp_b200 import FAP_DTYPE_F32, FAP_MODE_BATCHED, Context, DeviceGraph

pytestmark = pytest.mark.gpu


def _dg(case):
    ctx = Context(0)
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
    dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"],
                 case["bdy_num"])
    return ctx, dg


def _blocks(dg, parts):
    return {p: dg.copy_block(p, out_dtype=FAP_DTYPE_F32) for p in parts}


def _bits_equal(a, b):
    assert a.shape == b.shape
    np.testing.assert_array_equal(a.view(np.int32), b.view(np.int32))


def _has_duplicate_arcs(case):
    ro, col = case["row_offset"], case["col_val"]
    return any(len(set(col[ro[u]:ro[u + 1]].tolist())) != ro[u + 1] - ro[u]
               for u in range(len(ro) - 1))


@pytest.mark.parametrize("per_cta", [0, 1])
@pytest.mark.parametrize("name", golden_names())
def test_cached_solve_is_identical(cuda_ok, name, per_cta):
    case = load_golden(name)
    K = int(case["K"])
    vn = case["ver_num"]
    ctx, dg = _dg(case)
    dg.set_param("floyd_per_cta", per_cta)
    dg.solve(mode=FAP_MODE_BATCHED)
    ref = _blocks(dg, range(1, K + 1))
    est, built = dg.cache_bytes()
    assert not built and est > 0
    dg.cache_build()
    dg.check()
    held, built = dg.cache_bytes()
    assert built and 0 < held <= est
    dg.solve(mode=FAP_MODE_BATCHED)
    got = _blocks(dg, range(1, K + 1))
    for p in range(1, K + 1):
        _bits_equal(got[p], ref[p])
    if "row_checksums" in case:
        cs = np.concatenate([dg.block_checksums(p) for p in range(1, K + 1)])
        np.testing.assert_array_equal(cs, case["row_checksums"])
    # packed placement of a subset, cached and with the cache switched off
    sub = sorted({K, 1})
    dg.reserve(int(sum(vn[p] for p in sub)))
    dg.solve(sub, mode=FAP_MODE_BATCHED)
    for p, blk in _blocks(dg, sub).items():
        _bits_equal(blk, ref[p])
    dg.set_param("use_cache", 0)
    dg.solve(sub, mode=FAP_MODE_BATCHED)
    for p, blk in _blocks(dg, sub).items():
        _bits_equal(blk, ref[p])
    # the cache survives releasing the outputs; a new partition drops it
    dg.set_param("use_cache", 1)
    dg.release()
    assert dg.cache_bytes()[1]
    dg.solve([1], mode=FAP_MODE_BATCHED)
    _bits_equal(dg.copy_block(1, out_dtype=FAP_DTYPE_F32), ref[1])
    dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"],
                 case["bdy_num"])
    assert not dg.cache_bytes()[1]


@pytest.mark.parametrize("name", golden_names())
def test_cached_rows_equal_block_rows(cuda_ok, name):
    case = load_golden(name)
    K, n = int(case["K"]), int(case["n"])
    ctx, dg = _dg(case)
    rng = np.random.default_rng(3)
    src = rng.integers(0, n, size=min(3 * n, 300)).tolist() + [0, n - 1, 0]
    sssp = dg.rows(src)                       # no cache: SSSP rows
    dg.solve(mode=FAP_MODE_BATCHED)
    blocks = _blocks(dg, range(1, K + 1))
    dg.cache_build()
    cached = dg.rows(src)
    ed2st = np.empty(n, np.int64)
    ed2st[case["st2ed"]] = np.arange(n)
    for r, v in enumerate(src):
        p = int(case["graph_id"][v])
        i = int(ed2st[v] - case["ver_offset"][p])
        _bits_equal(cached[r], blocks[p][i])
    if not _has_duplicate_arcs(case):     # duplicates: the block keeps the last arc
        if case["integral"]:
            _bits_equal(cached, sssp)
        else:
            reach = sssp < 1e8
            assert np.array_equal(reach, cached < 1e8)
            rel = np.abs(cached[reach] - sssp[reach]) / np.maximum(np.abs(sssp[reach]), 1e-30)
            assert rel.max(initial=0.0) <= 1e-5
