"""The packed 16-bit min-plus tiles (int32 graphs, parts with more than 16
boundary vertices) give the same int32 blocks as the int32 tiles, whether
all, some or none of the tiles fit the packed form, in the plain, the
batched and the cached solves, and with the operands packed beforehand
("minplus_prepack" 1, the default) or stage by stage in shared memory (0)."""
import numpy as np
import pytest

from fastapsp_b200 import FAP_MODE_BATCHED, FAP_MODE_PLAIN, Context, DeviceGraph, fapGraph
from fastapsp_b200 import generators as G

pytestmark = pytest.mark.gpu


def _device_graph(el, K, tmp, name):
    G.write_mtx(el, tmp, name)
    g = fapGraph(name, el.directed, el.weighted, K, root=str(tmp))
    g.preCondition()
    ro, col, w = g.csr()
    vn, vo, bn = g.partInfo()
    dg = DeviceGraph(Context(0), ro, col, w)
    dg.set_parts(K, g.getGraphId(), g.getMapping(), vn, vo, bn)
    return dg, vn, bn


def _blocks(dg, parts):
    return [dg.copy_block(p) for p in parts]


def _grid(heavy_rows, heavy_wmax, seed):
    """96 x 96 grid, weights 1..100, but 1..heavy_wmax on the edges of the
    rows at or below heavy_rows: parts there have distances too long for the
    packed form."""
    el = G.grid_graph(96, 96, extra_frac=0.01, wmin=1, wmax=100, seed=seed)
    rng = np.random.default_rng(seed)
    heavy = (el.edges // 96 >= heavy_rows).all(axis=1)
    el.weights = el.weights.copy()
    el.weights[heavy] = rng.integers(1, heavy_wmax + 1, int(heavy.sum())).astype(np.float32)
    return el


@pytest.mark.parametrize("prepack", [1, 0])
@pytest.mark.parametrize("heavy_rows,expect", [(96, "all"), (48, "some"), (0, "none")])
def test_packed_tiles_equal_int32_tiles(cuda_ok, tmp_path, heavy_rows, expect, prepack):
    el = _grid(heavy_rows, 200000, 11)
    dg, vn, bn = _device_graph(el, 12, tmp_path, f"pk{heavy_rows}")
    dg.set_param("minplus_prepack", prepack)
    parts = list(range(1, 13))
    assert int(bn[1:].min()) > 16          # every part runs the min-plus tile kernel
    dg.set_param("minplus_pack16", 0)
    dg.solve(parts, FAP_MODE_BATCHED)
    ref = _blocks(dg, parts)
    assert dg.pack16_tiles() == (0, 0)
    dg.set_param("minplus_pack16", 1)
    for mode in (FAP_MODE_BATCHED, FAP_MODE_PLAIN):
        dg.solve(parts, mode)
        for p, want in zip(parts, ref):
            got = dg.copy_block(p)
            assert np.array_equal(got, want), f"part {p} mode {mode}"
    packed, total = dg.pack16_tiles()
    assert total > 0
    if expect == "all":
        assert packed == total
    elif expect == "none":
        assert packed == 0
    else:
        assert 0 < packed < total, (packed, total)


@pytest.mark.parametrize("prepack", [1, 0])
def test_packed_tiles_from_the_resident_cache(cuda_ok, tmp_path, prepack):
    el = G.grid_graph(96, 96, extra_frac=0.01, wmin=1, wmax=100, seed=12)
    dg, vn, bn = _device_graph(el, 12, tmp_path, "pkc")
    dg.set_param("minplus_prepack", prepack)
    dg.set_param("minplus_pack16", 0)
    dg.solve(None, FAP_MODE_BATCHED)
    ref = _blocks(dg, range(1, 13))
    dg.set_param("minplus_pack16", 1)
    dg.cache_build()
    dg.reserve(int(sum(vn[p] for p in (2, 5, 9))))
    dg.solve([2, 5, 9], FAP_MODE_BATCHED)
    for p in (2, 5, 9):
        assert np.array_equal(dg.copy_block(p), ref[p - 1]), f"part {p}"
    assert dg.pack16_tiles()[0] > 0


@pytest.mark.parametrize("prepack", [1, 0])
@pytest.mark.parametrize("heavy_rows", [96, 48])
def test_packed_expansion_tiles_equal_int32(cuda_ok, prepack, heavy_rows):
    """The tiled expansion of the boundary graph (Bellman-Ford closure, forced
    on a small grid) in packed 16-bit tiles gives the int32 tiles' blocks,
    with the operands packed beforehand or stage by stage, whether every or
    only some of the tiles fit."""
    el = _grid(heavy_rows, 200000, 13)
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        dg, vn, bn = _device_graph(el, 12, tmp, "pkx")
    dg.set_param("minplus_prepack", prepack)
    dg.set_param("bgraph_form", 2)
    dg.set_param("minplus_pack16", 0)
    dg.solve(None, FAP_MODE_BATCHED)
    assert "Bellman-Ford" in dg.stage1_name()
    ref = _blocks(dg, range(1, 13))
    assert dg.expand16_tiles() == (0, 0)
    dg.set_param("minplus_pack16", 1)
    dg.solve(None, FAP_MODE_BATCHED)
    for p in range(1, 13):
        assert np.array_equal(dg.copy_block(p), ref[p - 1]), f"part {p}"
    packed, total = dg.expand16_tiles()
    assert 0 < packed <= total
    dg.cache_build()                  # the cache build's expansion
    dg.solve(None, FAP_MODE_BATCHED)
    for p in range(1, 13):
        assert np.array_equal(dg.copy_block(p), ref[p - 1]), f"part {p} (cache)"


@pytest.mark.parametrize("thin_max_b", [0, 4, 8])
def test_thin_threshold_changes_no_value(cuda_ok, thin_max_b):
    """Parts with few boundary vertices in the register-tiled (packed) min-plus
    instead of the thin kernel give the same blocks (the autotuner's third
    choice)."""
    from fastapsp_b200 import workloads
    wl = workloads.load("road20k")
    ro, col, w = wl.csr()
    dg = DeviceGraph(Context(0), ro, col, w)
    dg.set_parts(wl.K, wl.graph.getGraphId(), wl.graph.getMapping(), wl.ver_num, wl.ver_offset, wl.bdy_num)
    dg.solve(None, FAP_MODE_BATCHED)
    want = _blocks(dg, range(1, wl.K + 1))
    dg.set_param("thin_max_b", thin_max_b)
    for mode in (FAP_MODE_BATCHED, FAP_MODE_PLAIN):
        dg.solve(None, mode)
        for p in range(1, wl.K + 1):
            assert np.array_equal(dg.copy_block(p), want[p - 1]), f"part {p} mode {mode}"
