"""GPU parity on mid-size graphs where the automatic rules pick the forms the
small fixtures reach only when forced, against fixtures the reference binary
made (tests/golden/make_golden_mid.py):

  road20k  int32    boundary graph closed by Floyd, thin min-plus
  grid256  int32    boundary graph over more than 8,192 boundary vertices:
                    Bellman-Ford closure and tiled expansion, min-plus tiles;
                    also solved in groups of parts from the resident cache
  rmat14   float32  tiled multi-source Bellman-Ford SSSP (directed, m >= 6n)

The graphs are regenerated from their seeds; the partition and renumbering
must equal the fixture's (which equal the reference's).  int32: every row's
checksum bit-exact; float32: sampled rows within |d - ref| <= 1e-5 |ref|,
reachability exact."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from fastapsp_b200 import FAP_MODE_BATCHED, Context, DeviceGraph, workloads

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5
MID = os.path.join(GOLDEN, "mid")


def _case(name):
    z = np.load(os.path.join(MID, name + ".npz"))
    return {k: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files}


def _graph(name):
    case = _case(name)
    wl = workloads.load(name)
    assert np.array_equal(wl.graph.getGraphId(), case["graph_id"]), "partition differs"
    assert np.array_equal(wl.graph.getMapping(), case["st2ed"]), "renumbering differs"
    ctx = Context(0)
    ro, col, w = wl.csr()
    dg = DeviceGraph(ctx, ro, col, w)
    dg.set_parts(wl.K, case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"],
                 case["bdy_num"])
    return case, wl, ctx, dg


def _checksums(dg, parts):
    return np.concatenate([dg.block_checksums(p) for p in parts])


@pytest.mark.parametrize("name,stage1", [("road20k", "boundary graph, Floyd"),
                                         ("grid256", "boundary graph, Bellman-Ford")])
def test_midsize_int32_matches_reference_checksums(cuda_ok, name, stage1):
    case, wl, ctx, dg = _graph(name)
    K = wl.K
    dg.solve(None, FAP_MODE_BATCHED)
    assert stage1 in dg.stage1_name(), dg.stage1_name()
    got = _checksums(dg, range(1, K + 1))
    bad = np.flatnonzero(got != case["row_checksums"])
    assert bad.size == 0, f"{bad.size} rows differ, first {bad[:5].tolist()}"


def test_grid256_grouped_from_the_cache_matches_reference(cuda_ok):
    """A job solved in groups of parts: stages 1-2 of every part once into
    the resident cache, then each group's min-plus merge from it."""
    case, wl, ctx, dg = _graph("grid256")
    K = wl.K
    vn = case["ver_num"]
    dg.cache_build()
    dg.check()
    groups = [list(range(a, min(a + 9, K + 1))) for a in range(1, K + 1, 9)]
    dg.reserve(max(int(sum(vn[p] for p in g)) for g in groups))
    got = []
    for g in groups:
        dg.solve(g, FAP_MODE_BATCHED)
        got.append(_checksums(dg, g))
    got = np.concatenate(got)
    bad = np.flatnonzero(got != case["row_checksums"])
    assert bad.size == 0, f"{bad.size} rows differ, first {bad[:5].tolist()}"


def test_rmat14_float32_matches_reference_rows(cuda_ok):
    case, wl, ctx, dg = _graph("rmat14")
    dg.solve(None, FAP_MODE_BATCHED)
    assert "Bellman-Ford" in dg.stage1_name(), dg.stage1_name()
    vo, vn = case["ver_offset"], case["ver_num"]
    n = wl.n
    rows = case["sample_rows"]
    for p in range(1, wl.K + 1):
        blk = dg.copy_block(p)
        assert blk.shape == (vn[p], n)
        for r, ref in zip(rows, case["sample_dist"]):
            if vo[p] <= r < vo[p] + vn[p]:
                got = blk[r - vo[p]]
                reach = ref < 1e8
                assert np.array_equal(reach, got < 1e8), f"row {r}: reachability differs"
                rel = np.abs(got[reach].astype(np.float64) - ref[reach]) / np.maximum(np.abs(ref[reach]), 1e-30)
                assert rel.max(initial=0.0) <= REL_TOL, (r, float(rel.max()))
