"""GPU parity: the CUDA path, called through the C ABI, against the reference's
outputs (committed golden fixtures made by the reference itself) and against
the oracle (C restatement) on seeded inputs.

Tolerances: int32 distances bit-exact (including the 1e8 sentinel); float32
distances |d - ref| <= 1e-5 * |ref| with reachability (== 1e8) exact.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_names, load_golden, write_golden_mtx
from fastapsp_b200 import (FAP_DTYPE_F32, FAP_DTYPE_I32, FAP_MODE_BATCHED, FAP_MODE_PLAIN,
                           Context, DeviceGraph, FapError, fapGraph)
from fastapsp_b200 import _lib as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5


def assert_dist_equal(got, ref, integral):
    got = np.asarray(got, np.float32)
    ref = np.asarray(ref, np.float32)
    assert got.shape == ref.shape
    if integral:
        bad = np.argwhere(got.view(np.int32) != ref.view(np.int32))
        assert bad.size == 0, f"{len(bad)} mismatches, first {bad[:5].tolist()}"
    else:
        reach = ref < 1e8
        assert np.array_equal(reach, got < 1e8), "reachability differs"
        rel = np.abs(got[reach] - ref[reach]) / np.maximum(np.abs(ref[reach]), 1e-30)
        assert rel.max(initial=0.0) <= REL_TOL, rel.max()


def build_graph(case, tmp, mode, dtype=None):
    write_golden_mtx(case, tmp)
    g = fapGraph(case["name"], bool(case["directed"]), bool(case["weighted"]), int(case["K"]),
                 root=tmp)
    if case["injected_partition"]:
        gid0 = (np.arange(case["n"], dtype=np.int64) * case["K"] // case["n"]).astype(np.int32)
        g.setPartition(gid0 + 1)
    g.setOptions(mode=mode, dtype=dtype)
    g.preCondition()
    return g


@pytest.mark.parametrize("mode", [FAP_MODE_BATCHED, FAP_MODE_PLAIN])
@pytest.mark.parametrize("name", golden_names())
def test_solve_matches_reference(cuda_ok, name, mode):
    case = load_golden(name)
    with tempfile.TemporaryDirectory() as tmp:
        g = build_graph(case, tmp, mode)
        assert g.dtype() == (FAP_DTYPE_I32 if case["integral"] else FAP_DTYPE_F32)
        if "dist" in case:
            assert g.solve() == 0
            assert_dist_equal(g.getAllDistance(), case["dist"], case["integral"])
        else:
            n = case["n"]
            cs = []
            for p in range(1, case["K"] + 1):
                assert g.solveSubGraph(p) == 0
                blk = g.getSubGraphDistance(p)
                assert blk.shape == (case["ver_num"][p], n)
                cs.append(O.row_checksums(O.to_i32(blk)))
                off = case["ver_offset"][p]
                for r, row in zip(case["sample_rows"], case["sample_dist"]):
                    if off <= r < off + blk.shape[0]:
                        assert_dist_equal(blk[r - off], row, True)
            np.testing.assert_array_equal(np.concatenate(cs), case["row_checksums"])


@pytest.mark.parametrize("name", ["grid12_k4", "road300_k6", "rmat8_int_k4"])
def test_float_path_on_integer_graph(cuda_ok, name):
    """Forcing float32 distances on integer weights must give the same values
    (every distance is below 2^24, so float sums are exact)."""
    case = load_golden(name)
    with tempfile.TemporaryDirectory() as tmp:
        g = build_graph(case, tmp, FAP_MODE_BATCHED, dtype=FAP_DTYPE_F32)
        assert g.dtype() == FAP_DTYPE_F32
        g.solve()
        assert_dist_equal(g.getAllDistance(), case["dist"], True)


def test_subgraph_getters_and_self_check(cuda_ok):
    case = load_golden("road300_k6")
    with tempfile.TemporaryDirectory() as tmp:
        g = build_graph(case, tmp, FAP_MODE_BATCHED)
        n = case["n"]
        for p in (1, 4):
            g.solveSubGraph(p)
            assert g.getCurrentSubGraphId() == p
            blk = g.getSubGraphDistance(p)
            off = case["ver_offset"][p]
            assert_dist_equal(blk, case["dist"][off:off + blk.shape[0]], True)
            idx = g.getSubGraphIndex(p)
            v = int(idx[3])
            row = g.getDistanceFromOnePoint(v)
            assert_dist_equal(row, blk[3], True)
            assert g.getDistanceP2P(v, 7) == blk[3, 7]
        with pytest.raises(FapError):
            g.getSubGraphDistance(1)  # not the current part


@pytest.mark.parametrize("mode", [FAP_MODE_BATCHED, FAP_MODE_PLAIN])
@pytest.mark.parametrize("name", ["road300_k6", "rmat8_f32_k4", "grid12_k4"])
def test_bounded_resident_rows_match_reference(cuda_ok, name, mode):
    """With fewer output rows allowed on the device than the graph has (as
    when HBM cannot hold all n rows), solveSubGraph and solve run the parts
    in groups that fit (in the batched form from the resident cache) and
    give the reference's values; a part with more rows than the bound is
    refused."""
    case = load_golden(name)
    K, vn, vo = case["K"], case["ver_num"], case["ver_offset"]
    with tempfile.TemporaryDirectory() as tmp:
        g = build_graph(case, tmp, mode)
        g.setMaxResidentRows(2 * int(max(vn[1:])))
        for p in list(range(K, 0, -1)) + [1, 2, 1]:
            assert g.solveSubGraph(p) == 0
            assert_dist_equal(g.getSubGraphDistance(p), case["dist"][vo[p]:vo[p] + vn[p]],
                              case["integral"])
        if mode == FAP_MODE_BATCHED:
            assert g.device_graph().last_stage1() == 3  # from the resident cache
        assert g.solve() == 0
        assert_dist_equal(g.getAllDistance(), case["dist"], case["integral"])
        big = int(np.argmax(vn[1:])) + 1
        g.setMaxResidentRows(int(vn[big]) - 1)
        with pytest.raises(FapError):
            g.solveSubGraph(big)
        with pytest.raises(FapError):
            g.solve()
        g.setMaxResidentRows(0)
        assert g.solve() == 0
        assert_dist_equal(g.getAllDistance(), case["dist"], case["integral"])


@pytest.mark.parametrize("name", ["grid12_k4", "disconnected_k3"])
def test_check_result_self_check(cuda_ok, name):
    """check_result compares sampled entries with fresh GPU shortest-path rows
    (the reference's check_ans, fap/utils/checkResult.h:38-82).  Like the
    reference's, it expects true shortest distances, so graphs whose inner
    rows carry the duplicate-edge rule are excluded."""
    case = load_golden(name)
    with tempfile.TemporaryDirectory() as tmp:
        g = build_graph(case, tmp, FAP_MODE_BATCHED)
        for p in range(1, case["K"] + 1):
            g.solveSubGraph(p)
            assert g.check_result(p)


def test_plain_and_batched_blocks_identical(cuda_ok):
    case = load_golden("grid64_k8")
    with tempfile.TemporaryDirectory() as tmp:
        write_golden_mtx(case, tmp)
        ctx = Context(0)
        ro, col, w = case["row_offset"], case["col_val"], case["weight"]
        dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
        dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"],
                     case["ver_offset"], case["bdy_num"])
        dg.solve(mode=FAP_MODE_BATCHED)
        a = [dg.block_checksums(p) for p in range(1, case["K"] + 1)]
        dg.solve(mode=FAP_MODE_PLAIN)
        b = [dg.block_checksums(p) for p in range(1, case["K"] + 1)]
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(np.concatenate(a), case["row_checksums"])
        dg.set_param("cuda_graph", 0)      # direct launches instead of the captured graph
        dg.solve(mode=FAP_MODE_BATCHED)
        c0 = [dg.block_checksums(p) for p in range(1, case["K"] + 1)]
        np.testing.assert_array_equal(np.concatenate(c0), case["row_checksums"])
        dg.set_param("cuda_graph", 1)
        for _ in range(2):                  # replays of the captured graph
            dg.solve(mode=FAP_MODE_BATCHED)
        c1 = [dg.block_checksums(p) for p in range(1, case["K"] + 1)]
        np.testing.assert_array_equal(np.concatenate(c1), case["row_checksums"])
        t = dg.last_timing()            # stage events recorded inside the graph
        assert t[4] > 0 and np.all(t[:4] >= 0) and abs(t[:4].sum() - t[4]) < 0.05 * t[4] + 0.05
        dg.set_param("floyd_per_cta", 1)   # the one-CTA-per-part Floyd form
        dg.solve(mode=FAP_MODE_BATCHED)
        c = [dg.block_checksums(p) for p in range(1, case["K"] + 1)]
        np.testing.assert_array_equal(np.concatenate(c), case["row_checksums"])
        dg.set_param("floyd_per_cta", 0)
        # packed placement: only part 5 and 2, in a 2-part row budget
        dg.reserve(int(case["ver_num"][5] + case["ver_num"][2]))
        dg.solve([5, 2], mode=FAP_MODE_BATCHED)
        np.testing.assert_array_equal(dg.block_checksums(5), a[4])
        np.testing.assert_array_equal(dg.block_checksums(2), a[1])
        with pytest.raises(FapError):
            dg.block_info(1)   # not resident


def test_sssp_round_bound_reports_error_and_context_survives(cuda_ok):
    case = load_golden("grid64_k8")
    ctx = Context(0)
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
    dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"],
                 case["ver_offset"], case["bdy_num"])
    dg.set_param("stage1", 1)          # the SSSP form (the boundary-graph form has no rounds)
    dg.set_param("sssp_max_rounds", 3)
    with pytest.raises(FapError) as e:
        dg.solve(mode=FAP_MODE_BATCHED)
    assert e.value.code == L.FAP_ERR_NOT_CONVERGED
    dg.set_param("sssp_max_rounds", 0)
    dg.solve(mode=FAP_MODE_BATCHED)   # same context, same graph: works again
    cs = np.concatenate([dg.block_checksums(p) for p in range(1, case["K"] + 1)])
    np.testing.assert_array_equal(cs, case["row_checksums"])


def test_partition_with_a_cross_arc_end_outside_the_boundary_block_is_refused(cuda_ok):
    """A part's last boundary vertex counted as inner (bdy_num one short):
    set_parts refuses it before any device work, and the true partition is
    accepted on the same graph afterwards."""
    case = load_golden("grid12_k4")
    ctx = Context(0)
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
    bn = np.array(case["bdy_num"], copy=True)
    p = int(np.argmax(bn[1:])) + 1
    bn[p] -= 1
    with pytest.raises(FapError) as e:
        dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"], bn)
    assert e.value.code == L.FAP_ERR_PARTITION
    dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"],
                 case["bdy_num"])
    dg.solve(mode=FAP_MODE_BATCHED)
    for q in range(1, case["K"] + 1):
        off = int(case["ver_offset"][q])
        blk = dg.copy_block(q, out_dtype=FAP_DTYPE_F32)
        assert_dist_equal(blk, case["dist"][off:off + blk.shape[0]], True)


def test_sssp_delta_stepping_same_result(cuda_ok):
    case = load_golden("road300_k6")
    ctx = Context(0)
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
    src = list(range(0, 300, 7))
    base = dg.sssp_rows(src)
    for delta in (1, 50, 700, 5000):
        dg.set_param("sssp_delta", delta)
        np.testing.assert_array_equal(dg.sssp_rows(src), base)
    for i, s in enumerate(src):
        assert_dist_equal(base[i], O.port_dijkstra(ro, col, w, s), True)


# ---------------------------------------------------------------------------
# stage operators against the oracle / numpy
# ---------------------------------------------------------------------------
def _np_minplus(A, B, inf):
    A = A.astype(np.int64) if A.dtype == np.int32 else A
    B = B.astype(np.int64) if B.dtype == np.int32 else B
    M, K = A.shape
    N = B.shape[1]
    C = np.full((M, N), inf, A.dtype)
    for k in range(K):
        C = np.minimum(C, A[:, k:k + 1] + B[k:k + 1, :])
    return C


@pytest.mark.parametrize("shape", [(1, 1, 1), (5, 7, 0), (37, 45, 3), (128, 128, 16),
                                   (129, 257, 33), (300, 131, 97), (64, 1000, 11)])
@pytest.mark.parametrize("dtype", [FAP_DTYPE_I32, FAP_DTYPE_F32])
def test_op_minplus(cuda_ok, shape, dtype):
    import torch
    M, N, K = shape
    rng = np.random.default_rng(M * 1000 + N + K)
    if dtype == FAP_DTYPE_I32:
        A = rng.integers(0, 5000, (M, K)).astype(np.int32)
        B = rng.integers(0, 5000, (K, N)).astype(np.int32)
        A[rng.random((M, K)) < 0.2] = L.FAP_INF_I32
        B[rng.random((K, N)) < 0.2] = L.FAP_INF_I32
        ref = np.minimum(_np_minplus(A, B, L.FAP_INF_I32), L.FAP_INF_I32).astype(np.int32)
        tdt = torch.int32
    else:
        A = (rng.random((M, K)) * 100).astype(np.float32)
        B = (rng.random((K, N)) * 100).astype(np.float32)
        A[rng.random((M, K)) < 0.2] = 1e8
        B[rng.random((K, N)) < 0.2] = 1e8
        ref = np.minimum(_np_minplus(A, B, np.float32(1e8)), np.float32(1e8))
        tdt = torch.float32
    ctx = Context(0)
    ctx.use_torch_stream()
    dA = torch.from_numpy(A).cuda() if K else torch.empty((M, 1), dtype=tdt, device="cuda")
    dB = torch.from_numpy(B).cuda() if K else torch.empty((1, N), dtype=tdt, device="cuda")
    dC = torch.empty((M, N), dtype=tdt, device="cuda")
    if K == 0:
        dA = dA[:, :0]
        dB = dB[:0, :]
    ctx.minplus(dA, dB, dC, dtype)
    torch.cuda.synchronize()
    got = dC.cpu().numpy()
    assert np.array_equal(got.view(np.int32), ref.view(np.int32))


@pytest.mark.parametrize("s", [1, 5, 127, 128, 129, 300])
@pytest.mark.parametrize("dtype", [FAP_DTYPE_I32, FAP_DTYPE_F32])
def test_op_floyd(cuda_ok, s, dtype):
    import torch
    rng = np.random.default_rng(s)
    if dtype == FAP_DTYPE_I32:
        M = rng.integers(1, 1000, (s, s)).astype(np.float32)
    else:
        M = (np.exp(rng.uniform(np.log(0.01), np.log(100), (s, s)))).astype(np.float32)
    M[rng.random((s, s)) < 0.9] = 1e8
    np.fill_diagonal(M, 0)
    ref = O.port_floyd(M)
    ctx = Context(0)
    ctx.use_torch_stream()
    if dtype == FAP_DTYPE_I32:
        d = torch.from_numpy(M.astype(np.int32)).cuda()
    else:
        d = torch.from_numpy(M).cuda()
    ctx.floyd(d, dtype)
    torch.cuda.synchronize()
    got = d.cpu().numpy().astype(np.float32)
    assert_dist_equal(got, ref, dtype == FAP_DTYPE_I32)


@pytest.mark.parametrize("dtype", [FAP_DTYPE_I32, FAP_DTYPE_F32])
def test_op_sssp(cuda_ok, dtype):
    import torch
    from fastapsp_b200 import generators as G
    g = G.rmat_graph(10, 8000, seed=7) if dtype == FAP_DTYPE_F32 else G.road_graph(2000, seed=7)
    n = g.n
    src = np.repeat(g.edges[:, 0], 1 if g.directed else 2)
    if g.directed:
        a, b = g.edges[:, 0], g.edges[:, 1]
        w = g.weights
    else:
        a = np.concatenate([g.edges[:, 0], g.edges[:, 1]])
        b = np.concatenate([g.edges[:, 1], g.edges[:, 0]])
        w = np.concatenate([g.weights, g.weights])
    order = np.argsort(a, kind="stable")
    col = b[order].astype(np.int32)
    ww = w[order].astype(np.float32)
    ro = np.zeros(n + 1, np.int32)
    np.add.at(ro, a + 1, 1)
    ro = np.cumsum(ro).astype(np.int32)
    sources = np.array([0, 5, 17, n - 1], np.int32)
    ctx = Context(0)
    ctx.use_torch_stream()
    tw = torch.from_numpy(ww.astype(np.int32) if dtype == FAP_DTYPE_I32 else ww).cuda()
    out = torch.empty((len(sources), n + 3),
                      dtype=torch.int32 if dtype == FAP_DTYPE_I32 else torch.float32,
                      device="cuda")
    ctx.sssp(torch.from_numpy(ro).cuda(), torch.from_numpy(col).cuda(), tw,
             torch.from_numpy(sources).cuda(), out, dtype)
    torch.cuda.synchronize()
    got = out.cpu().numpy()[:, :n].astype(np.float32)
    for i, s in enumerate(sources):
        assert_dist_equal(got[i], O.port_dijkstra(ro, col, ww, int(s)), dtype == FAP_DTYPE_I32)


def test_legacy_abi_matches_oracle(cuda_ok):
    """The reference's own kernel ABI, called with host arrays."""
    import ctypes
    lib = L.lib()
    f_floyd = getattr(lib, L.LEGACY_SYMBOLS["floyd_GPU_Nvidia_path"])
    f_mp = getattr(lib, L.LEGACY_SYMBOLS["minplus_NVIDIA_path"])
    f_bd = getattr(lib, L.LEGACY_SYMBOLS["handle_boundry_Nvidia_GPU"])
    rng = np.random.default_rng(3)
    s = 70
    M = rng.integers(1, 50, (s, s)).astype(np.float32)
    M[rng.random((s, s)) < 0.85] = 1e8
    np.fill_diagonal(M, 0)
    ref = O.port_floyd(M)
    arc = M.copy()
    path = np.zeros((s, s), np.int32)
    f_floyd(ctypes.c_int(s), L.ptr(arc), L.ptr(path))
    assert lib.fap_legacy_last_status() == 0
    assert_dist_equal(arc, ref, True)
    m_, n_, k_ = 33, 50, 9
    A = rng.integers(0, 100, (m_, k_)).astype(np.float32)
    B = rng.integers(0, 100, (k_, n_)).astype(np.float32)
    res = np.zeros((m_, n_), np.float32)
    f_mp(L.ptr(A), L.ptr(B), L.ptr(np.zeros((k_, n_), np.int32)), L.ptr(res),
         L.ptr(np.zeros((m_, n_), np.int32)), m_, n_, k_)
    assert np.array_equal(res, _np_minplus(A, B, np.float32(1e8)))
    case = load_golden("road300_k6")
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    st2ed = case["st2ed"].astype(np.int32)
    off, b = int(case["ver_offset"][2]), int(case["bdy_num"][2])
    sub = np.zeros((b, case["n"]), np.float32)
    f_bd(L.ptr(sub), case["n"], case["m"], b, L.ptr(np.diff(ro).astype(np.int32)), L.ptr(ro),
         L.ptr(col), L.ptr(w), L.ptr(st2ed), off)
    assert lib.fap_legacy_last_status() == 0
    np.testing.assert_array_equal(sub, case["dist"][off:off + b])


def test_legacy_abi_blocked_floyd_entry_points(cuda_ok):
    """The rest of the reference's kernel header, which its fap/fap.cpp also
    calls: the blocked-Floyd column and row panels (fap/kernel/floyd.h:
    51-84, their CUDA versions from the sentinel), the remaining-block update
    res = min(res, mat1 (x) mat2) (:86-102), the path-free min-plus
    (minplus.h:69-76) and Floyd.  Integral inputs run in int32 and must match
    exactly; real-valued ones in float32 within the tolerance.  The path
    arrays given here are all zero, so they stay zero (predecessor outputs
    are tested in tests/test_legacy_paths.py)."""
    lib = L.lib()
    f = {k: getattr(lib, L.LEGACY_SYMBOLS[k]) for k in
         ("floyd_NVIDIA_GPU", "floyd_path_A_Nvidia", "floyd_path_B_Nvidia", "floyd_min_plus_Nvidia",
          "minplus_NVIDIA_GPU")}
    inf = np.float32(1e8)
    rng = np.random.default_rng(21)
    for integral in (True, False):
        def mat(r, c, p_inf=0.4):
            if integral:
                x = rng.integers(0, 60, (r, c)).astype(np.float32)
            else:
                x = (rng.random((r, c)) * 60).astype(np.float32)
            x[rng.random((r, c)) < p_inf] = inf
            return x

        def closed(s):
            d = mat(s, s, 0.7)
            np.fill_diagonal(d, 0)
            return O.port_floyd(d)

        row, col = 37, 23
        # Floyd without paths
        arc = mat(50, 50, 0.85)
        np.fill_diagonal(arc, 0)
        want = O.port_floyd(arc)
        f["floyd_NVIDIA_GPU"](50, L.ptr(arc))
        assert lib.fap_legacy_last_status() == 0
        assert_dist_equal(arc, want, integral)
        # column panel A[row x col] against diag[col x col]
        diag = closed(col)
        A = mat(row, col)
        want = _np_minplus(A, diag, inf)
        A_path, diag_path = np.zeros((row, col), np.int32), np.zeros((col, col), np.int32)
        f["floyd_path_A_Nvidia"](L.ptr(A), L.ptr(A_path), row, col, L.ptr(diag), L.ptr(diag_path))
        assert lib.fap_legacy_last_status() == 0
        assert_dist_equal(A, want, integral)
        assert not A_path.any()
        # row panel B[row x col] against diag[row x row]
        diag = closed(row)
        B = mat(row, col)
        want = _np_minplus(diag, B, inf)
        B_path, diag_path = np.zeros((row, col), np.int32), np.zeros((row, row), np.int32)
        f["floyd_path_B_Nvidia"](L.ptr(B), L.ptr(B_path), row, col, L.ptr(diag), L.ptr(diag_path))
        assert lib.fap_legacy_last_status() == 0
        assert_dist_equal(B, want, integral)
        # remaining blocks: res = min(res, mat1 (x) mat2), also with k = 0
        for m_, n_, k_ in ((29, 41, 13), (5, 9, 0)):
            m1, m2, res = mat(m_, k_), mat(k_, n_), mat(m_, n_, 0.3)
            want = np.minimum(res, _np_minplus(m1, m2, inf))
            f["floyd_min_plus_Nvidia"](L.ptr(m1), L.ptr(m2), L.ptr(np.zeros((k_, n_), np.int32)), L.ptr(res),
                                       L.ptr(np.zeros((m_, n_), np.int32)), m_, n_, k_)
            assert lib.fap_legacy_last_status() == 0
            assert_dist_equal(res, want, integral)
        # path-free min-plus from the sentinel (res's old values are ignored)
        m1, m2, res = mat(33, 19), mat(19, 47), np.zeros((33, 47), np.float32)
        f["minplus_NVIDIA_GPU"](L.ptr(m1), L.ptr(m2), L.ptr(res), 33, 47, 19)
        assert lib.fap_legacy_last_status() == 0
        assert_dist_equal(res, _np_minplus(m1, m2, inf), integral)


def test_relax_peak_is_positive(cuda_ok):
    ctx = Context(0)
    assert ctx.relax_peak(FAP_DTYPE_I32) > 1e12


@pytest.mark.parametrize("name", ["grid64_k8", "rmat8_f32_k4", "road300_k6"])
def test_async_block_copies_equal_the_synchronous_ones(cuda_ok, name):
    """fap_graph_copy_block_async on the two copy slots (float32 output, and
    the graph's own dtype without conversion) gives the bytes
    fap_graph_copy_block gives; a slot reused waits for its previous copy."""
    case = load_golden(name)
    K = int(case["K"])
    ctx = Context(0)
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
    dg.set_parts(K, case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"], case["bdy_num"])
    dg.solve(mode=FAP_MODE_BATCHED)
    dg.check()
    vn, n = case["ver_num"], int(case["n"])
    for dt in sorted({FAP_DTYPE_F32, dg.dtype}):
        want = {p: dg.copy_block(p, out_dtype=dt) for p in range(1, K + 1)}
        npdt = np.float32 if dt == FAP_DTYPE_F32 else np.int32
        outs = {p: np.full((int(vn[p]), n), -7, npdt) for p in range(1, K + 1)}
        for k, p in enumerate(range(1, K + 1)):
            dg.copy_block_async(p, outs[p], k % 2, out_dtype=dt)
        dg.copy_wait(0)
        dg.copy_wait(1)
        for p in range(1, K + 1):
            assert np.array_equal(outs[p].view(np.int32), want[p].view(np.int32)), (dt, p)
    with pytest.raises(FapError):  # (the last loop's buffers are float32)
        dg.copy_block_async(1, outs[1], 2, out_dtype=FAP_DTYPE_F32)
