"""Seeded random graphs through every form of the solve path, against the
oracle's restatement of fapGraph::run (fap/fap.cpp:92-181: Dijkstra from the
part's boundary vertices, the submatrix build, Floyd-Warshall, min-plus and
decode, per part; pinned to the reference binary in tests/test_oracle.py).

Families: road-shaped, grid with long-range edges, random geometric (all
undirected, integer weights: int32 distances, bit-exact) and directed R-MAT
with float weights (float32, |d - ref| <= 1e-5 |ref|, reachability exact).
The partition and renumbering come from this library's own host
preprocessing (METIS k-way, boundary detection, sort_and_encode); every case
is then solved with stage 1 by the frontier and the tiled SSSP, by the
boundary graph closed by Floyd and by Bellman-Ford, with the Floyd as the
work queue and as per-phase launches, symmetric and not, with thin and tile
min-plus kernels, packed (operands packed beforehand or per stage) and int32
tiles, in the plain form, and from the resident cache."""
import numpy as np
import pytest

from fastapsp_b200 import FAP_DTYPE_F32, FAP_MODE_BATCHED, FAP_MODE_PLAIN, Context, DeviceGraph, fapGraph
from fastapsp_b200 import generators as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5

CASES = [
    ("road", 600, 6, 0), ("road", 1500, 12, 1), ("road", 900, 3, 2),
    ("grid", 24, 5, 3), ("grid", 36, 9, 4),
    ("rgg", 1200, 8, 5),
    ("rmat", 9, 4, 6), ("rmat", 10, 6, 7),
]

FORMS = [
    {},                                            # automatic
    {"stage1": 1},                                 # frontier SSSP
    {"stage1": 1, "sssp_form": 2},                 # tiled SSSP
    {"stage1": 2},                                 # boundary graph (Floyd closure at these sizes)
    {"stage1": 2, "bgraph_form": 2},               # boundary graph, Bellman-Ford closure
    {"floyd_queue": 0},                            # per-phase Floyd launches
    {"floyd_symmetric": 0},                        # full Floyd items
    {"thin_max_b": 0},                             # register-tiled min-plus for every part
    {"thin_max_b": 0, "minplus_pack16": 0},        # ... in int32 only
    {"thin_max_b": 0, "minplus_prepack": 0},       # ... packed stage by stage in shared memory
]


def _edges(family, size, seed):
    if family == "road":
        return G.road_graph(size, seed=seed)
    if family == "grid":
        return G.grid_graph(size, size, drop_frac=0.05, extra_frac=0.01, wmin=1, wmax=100, seed=seed)
    if family == "rgg":
        return G.random_geometric_graph(size, 3.0, seed=seed)
    return G.rmat_graph(size, 8 << size, seed=seed)


@pytest.fixture(scope="module", params=CASES, ids=lambda c: f"{c[0]}{c[1]}_k{c[2]}_s{c[3]}")
def case(request):
    family, size, K, seed = request.param
    g = _edges(family, size, seed)
    ro, col, w = G.edges_to_csr(g)
    fg = fapGraph.from_csr(g.n, int(ro[-1]), ro, col, w, K, directed=g.directed)
    fg.preCondition()
    ro, col, w = fg.csr()
    gid = fg.getGraphId()
    st2ed = fg.getMapping()
    vn, vo, bn = fg.partInfo()
    ed2st = np.empty_like(st2ed)
    ed2st[st2ed] = np.arange(st2ed.shape[0], dtype=st2ed.dtype)
    want = {p: O.port_run_part(ro, col, w, gid, st2ed, ed2st, int(vo[p]), int(vn[p]), int(bn[p]))
            for p in range(1, K + 1)}
    return dict(n=g.n, K=K, ro=ro, col=col, w=w, gid=gid, st2ed=st2ed, vn=vn, vo=vo, bn=bn,
                integral=bool(g.integral), want=want)


def _check(dg, case):
    for p in range(1, case["K"] + 1):
        got = dg.copy_block(p, out_dtype=FAP_DTYPE_F32)
        ref = case["want"][p]
        if case["integral"]:
            bad = np.flatnonzero((got.view(np.int32) != ref.view(np.int32)).any(1))
            assert bad.size == 0, f"part {p}: rows {bad[:5].tolist()} differ"
        else:
            reach = ref < 1e8
            assert np.array_equal(reach, got < 1e8), f"part {p}: reachability differs"
            rel = np.abs(got[reach].astype(np.float64) - ref[reach]) / np.maximum(np.abs(ref[reach]), 1e-30)
            assert rel.max(initial=0.0) <= REL_TOL, (p, float(rel.max()))


def _device_graph(case):
    ctx = Context(0)
    dg = DeviceGraph(ctx, case["ro"], case["col"], case["w"])
    dg.set_parts(case["K"], case["gid"], case["st2ed"], case["vn"], case["vo"], case["bn"])
    return ctx, dg


@pytest.mark.parametrize("form", FORMS, ids=lambda f: ",".join(f"{k}={v}" for k, v in f.items()) or "auto")
def test_random_graph_batched_forms_match_oracle(cuda_ok, case, form):
    ctx, dg = _device_graph(case)
    for k, v in form.items():
        dg.set_param(k, v)
    dg.solve(mode=FAP_MODE_BATCHED)
    dg.check()
    _check(dg, case)


def test_random_graph_plain_and_cached_match_oracle(cuda_ok, case):
    ctx, dg = _device_graph(case)
    dg.solve(mode=FAP_MODE_PLAIN)
    dg.check()
    _check(dg, case)
    dg.cache_build()
    dg.check()
    dg.solve(mode=FAP_MODE_BATCHED)
    dg.check()
    assert dg.last_stage1() == 3
    _check(dg, case)
    # parts in groups from the cache, in reverse order
    K = case["K"]
    groups = [list(range(K, 0, -1))[i:i + 2] for i in range(0, K, 2)]
    dg.reserve(max(int(sum(case["vn"][p] for p in g)) for g in groups))
    for g in groups:
        dg.solve(g, FAP_MODE_BATCHED)
        dg.check()
        for p in g:
            got = dg.copy_block(p, out_dtype=FAP_DTYPE_F32)
            ref = case["want"][p]
            if case["integral"]:
                assert np.array_equal(got.view(np.int32), ref.view(np.int32)), p
            else:
                reach = ref < 1e8
                assert np.array_equal(reach, got < 1e8)
                rel = np.abs(got[reach].astype(np.float64) - ref[reach]) / np.maximum(np.abs(ref[reach]), 1e-30)
                assert rel.max(initial=0.0) <= REL_TOL
