"""The batched Floyd-Warshall as one persistent launch over a work queue
(parameter "floyd_queue", the default) against the three-launches-per-pivot
form: the same tile updates run in the same dependency order, so the blocks
are bit-identical (float32 too), in each form the queue takes:
  boundary-graph stage 1        Floyd items only (local closures); on
                                undirected graphs only the tiles on and
                                above the diagonal, each storing its
                                transpose (parameter "floyd_symmetric")
  SSSP stage 1, packed min-plus Floyd + boundary-row scatter items
  SSSP stage 1, int32 / float32 Floyd + scatter + min-plus tiles, one launch
  resident cache build          Floyd (+ scatter) items of every part"""
import numpy as np
import pytest

from fastapsp_b200 import FAP_MODE_BATCHED, Context, DeviceGraph, workloads

pytestmark = pytest.mark.gpu


def _dg(name):
    wl = workloads.load(name)
    ro, col, w = wl.csr()
    dg = DeviceGraph(Context(0), ro, col, w)
    dg.set_parts(wl.K, wl.graph.getGraphId(), wl.graph.getMapping(), wl.ver_num, wl.ver_offset, wl.bdy_num)
    return wl, dg


def _solve_all(dg, K, queue, **params):
    dg.set_param("floyd_queue", 1 if queue else 0)
    for k, v in params.items():
        dg.set_param(k, v)
    dg.solve(None, FAP_MODE_BATCHED)
    return [dg.copy_block(p) for p in range(1, K + 1)]


@pytest.mark.parametrize("name,params", [
    ("grid128", {}),                                           # boundary graph (int32)
    ("grid128", {"stage1": 1}),                                # SSSP form, packed min-plus
    ("grid128", {"stage1": 1, "minplus_pack16": 0}),           # SSSP form, min-plus in the queue
    ("rmat14", {}),                                            # float32, min-plus in the queue
    ("road20k", {}),                                           # thin parts only
])
def test_queue_equals_multi_launch(cuda_ok, name, params):
    wl, dg = _dg(name)
    want = _solve_all(dg, wl.K, False, **params)
    got = _solve_all(dg, wl.K, True, **params)
    for p, (a, b) in enumerate(zip(got, want), 1):
        assert np.array_equal(a.view(np.int32), b.view(np.int32)), f"part {p}"


@pytest.mark.parametrize("name", ["grid128", "rmat14"])
def test_queue_in_the_cache_build(cuda_ok, name):
    wl, dg = _dg(name)
    want = _solve_all(dg, wl.K, False)
    dg.set_param("floyd_queue", 1)
    dg.cache_build()
    dg.check()
    parts = [1, wl.K // 2, wl.K]
    dg.solve(parts, FAP_MODE_BATCHED)
    for p in parts:
        assert np.array_equal(dg.copy_block(p).view(np.int32), want[p - 1].view(np.int32)), f"part {p}"


@pytest.mark.parametrize("name", ["grid128", "road20k"])
def test_symmetric_queue_equals_full_queue(cuda_ok, name):
    """Undirected parts: the local closures are symmetric, and computing the
    upper tiles with their transposes gives the full computation's blocks."""
    wl, dg = _dg(name)
    want = _solve_all(dg, wl.K, True, floyd_symmetric=0)
    got = _solve_all(dg, wl.K, True, floyd_symmetric=1)
    assert "boundary graph" in dg.stage1_name()
    for p, (a, b) in enumerate(zip(got, want), 1):
        assert np.array_equal(a, b), f"part {p}"
