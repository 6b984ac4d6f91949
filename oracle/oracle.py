"""Oracle for the per-subgraph solve path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker or as the timed CPU baseline.  The product
(fastapsp_b200) never imports it.

Two oracles live here:

* the restatement ("port"): oracle/fap_oracle.c, a C restatement of the
  reference's CPU path, built as oracle/liboracle_port.so and called through
  ctypes below; plus numpy restatements of the host preprocessing
  (restate_boundary, restate_encode_classes);
* the reference itself ("ref"): oracle/_ref/fap_ref, the reference's own
  fap/fap.cpp compiled from its sources by oracle/Makefile, driven per part
  through fapGraph::run (fap/fap.cpp:92-181).

The port is pinned against the reference by tests/test_oracle.py and by the
committed fixtures under tests/golden/ (made by tests/golden/make_golden.py
from oracle/_ref).
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle_port.so")
REF_BIN = os.path.join(HERE, "_ref", "fap_ref")
MAXVALUE = np.float32(1e8)  # fap/utils/parameter.h:26


# --------------------------------------------------------------------------
# Reading the reference's CSR / partition / renumbering
# --------------------------------------------------------------------------

@dataclass
class Meta:
    """The reference's fapGraph state after preCondition (fap/fap.h:24-76):
    CSR, 1-based graph_id, st2ed/ed2st and per-part counts (index 1..K)."""
    n: int
    m: int
    K: int
    row_offset: np.ndarray
    col_val: np.ndarray
    weight: np.ndarray
    graph_id: np.ndarray
    st2ed: np.ndarray
    ed2st: np.ndarray
    ver_num: np.ndarray
    ver_offset: np.ndarray
    bdy_num: np.ndarray


def read_meta(path: str) -> Meta:
    """Parse the binary written by fap_ref --meta (see dump_meta there)."""
    raw = np.fromfile(path, dtype=np.int32)
    n, m, K = (int(x) for x in raw[:3])
    o = 3

    def take(cnt, dt=np.int32):
        nonlocal o
        a = raw[o:o + cnt].copy()
        o += cnt
        return a.view(dt) if dt is not np.int32 else a

    ro = take(n + 1)
    col = take(m)
    w = take(m, np.float32)
    gid = take(n)
    st2ed = take(n)
    ed2st = take(n)
    vn = take(K + 1)
    vo = take(K + 1)
    bn = take(K + 1)
    assert o == raw.size, "meta file size mismatch"
    return Meta(n, m, K, ro, col, w, gid, st2ed, ed2st, vn, vo, bn)


# --------------------------------------------------------------------------
# The C restatement
# --------------------------------------------------------------------------

_port = None


def port_lib():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            subprocess.run(["make", "-C", HERE, "port"], check=True,
                           stdout=subprocess.DEVNULL)
        lib = ctypes.CDLL(PORT_SO)
        P = ctypes.c_void_p
        I = ctypes.c_int
        lib.fo_run_part.argtypes = [I, P, P, P, P, P, P, I, I, I, P]
        lib.fo_run_part.restype = I
        lib.fo_dijkstra_path.argtypes = [I, I, P, P, P, P, P]
        lib.fo_dijkstra_path.restype = None
        lib.fo_floyd.argtypes = [I, P]
        lib.fo_floyd.restype = None
        lib.fo_floyd_path.argtypes = [I, P, P]
        lib.fo_floyd_path.restype = None
        lib.fo_minplus_path.argtypes = [I, I, I, P, P, P, P, P, P, P]
        lib.fo_minplus_path.restype = None
        lib.fo_floyd_path_A.argtypes = [P, P, I, I, P, P]
        lib.fo_floyd_path_A.restype = None
        lib.fo_floyd_path_B.argtypes = [P, P, I, I, P, P]
        lib.fo_floyd_path_B.restype = None
        _port = lib
    return _port


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def port_run_part(row_offset, col, weight, graph_id, st2ed, ed2st,
                  start: int, s: int, bdy: int) -> np.ndarray:
    """Solve one part with the C restatement of fapGraph::run; returns the
    s x n float32 block (row r = vertex st2ed[start + r], column = vertex id)."""
    n = int(row_offset.shape[0]) - 1
    ro = np.ascontiguousarray(row_offset, np.int32)
    cv = np.ascontiguousarray(col, np.int32)
    w = np.ascontiguousarray(weight, np.float32)
    gid = np.ascontiguousarray(graph_id, np.int32)
    s2e = np.ascontiguousarray(st2ed, np.int32)
    e2s = np.ascontiguousarray(ed2st, np.int32)
    out = np.empty((s, n), np.float32)
    rc = port_lib().fo_run_part(n, _p(ro), _p(cv), _p(w), _p(gid), _p(s2e), _p(e2s),
                                int(start), int(s), int(bdy), _p(out))
    if rc != 0:
        raise MemoryError("oracle part solve failed")
    return out


def port_dijkstra(row_offset, col, weight, src: int) -> np.ndarray:
    n = int(row_offset.shape[0]) - 1
    ro = np.ascontiguousarray(row_offset, np.int32)
    cv = np.ascontiguousarray(col, np.int32)
    w = np.ascontiguousarray(weight, np.float32)
    d = np.empty(n, np.float32)
    port_lib().fo_dijkstra_path(int(src), n, _p(ro), _p(cv), _p(w), _p(d), None)
    return d


def port_floyd(mat: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(mat, np.float32).copy()
    port_lib().fo_floyd(int(m.shape[0]), _p(m))
    return m


def port_floyd_path(mat: np.ndarray, path: np.ndarray):
    """floyd_CPU_path (fap/kernel/floyd.h:38-49): (closed matrix, paths)."""
    m = np.ascontiguousarray(mat, np.float32).copy()
    p = np.ascontiguousarray(path, np.int32).copy()
    port_lib().fo_floyd_path(int(m.shape[0]), _p(m), _p(p))
    return m, p


def port_minplus_path(mat1, mat2, mat2_path, c0=None, p0=None):
    """min_plus_path_CPU_advanced (fap/kernel/minplus.h:51-65) when c0 is
    None, floyd_min_plus_CPU (fap/kernel/floyd.h:86-102) from (c0, p0)
    otherwise: (values, paths)."""
    a = np.ascontiguousarray(mat1, np.float32)
    b = np.ascontiguousarray(mat2, np.float32)
    bp = np.ascontiguousarray(mat2_path, np.int32)
    M, K = a.shape
    N = b.shape[1]
    res = np.empty((M, N), np.float32)
    path = np.empty((M, N), np.int32)
    c0a = None if c0 is None else np.ascontiguousarray(c0, np.float32)
    p0a = None if c0 is None else np.ascontiguousarray(p0, np.int32)
    port_lib().fo_minplus_path(int(M), int(N), int(K), _p(a), _p(b), _p(bp),
                               None if c0a is None else _p(c0a), None if p0a is None else _p(p0a),
                               _p(res), _p(path))
    return res, path


def port_floyd_path_panel(which: str, panel, panel_path, diag, diag_path):
    """floyd_path_A_CPU / floyd_path_B_CPU (fap/kernel/floyd.h:51-84), in
    place like the reference: (values, paths)."""
    x = np.ascontiguousarray(panel, np.float32).copy()
    xp = np.ascontiguousarray(panel_path, np.int32).copy()
    d = np.ascontiguousarray(diag, np.float32)
    dp = np.ascontiguousarray(diag_path, np.int32)
    row, col = x.shape
    fn = port_lib().fo_floyd_path_A if which == "A" else port_lib().fo_floyd_path_B
    fn(_p(x), _p(xp), int(row), int(col), _p(d), _p(dp))
    return x, xp


def port_solve_meta(meta: Meta, parts=None) -> dict:
    """Solve the given 1-based parts of a Meta with the restatement."""
    out = {}
    parts = range(1, meta.K + 1) if parts is None else parts
    for p in parts:
        out[p] = port_run_part(meta.row_offset, meta.col_val, meta.weight, meta.graph_id,
                               meta.st2ed, meta.ed2st, int(meta.ver_offset[p]),
                               int(meta.ver_num[p]), int(meta.bdy_num[p]))
    return out


# --------------------------------------------------------------------------
# numpy restatements of the host preprocessing
# --------------------------------------------------------------------------

def restate_boundary(row_offset, col, graph_id) -> np.ndarray:
    """Boundary flags.  Follows fap/utils/util_preprocess.h:32-58
    (findBoundry): both endpoints of every out-edge whose endpoints lie in
    different parts are boundary."""
    n = row_offset.shape[0] - 1
    src = np.repeat(np.arange(n), np.diff(row_offset))
    cross = graph_id[src] != graph_id[col]
    flag = np.zeros(n, bool)
    flag[src[cross]] = True
    flag[col[cross]] = True
    return flag


def restate_encode_classes(graph_id, is_bdy, K):
    """What sort_and_encode (fap/utils/util_preprocess.h:73-106) guarantees,
    independent of how std::sort orders ties: per part p = 1..K the
    offset/count of its contiguous block, boundary vertices first, and the
    vertex set of every (part, boundary) class."""
    ver_num = np.zeros(K + 1, np.int64)
    bdy_num = np.zeros(K + 1, np.int64)
    np.add.at(ver_num, graph_id, 1)
    np.add.at(bdy_num, graph_id[is_bdy], 1)
    ver_off = np.zeros(K + 1, np.int64)
    ver_off[1:] = np.concatenate([[0], np.cumsum(ver_num[1:])[:-1]])
    return ver_num, ver_off, bdy_num


def check_encoding(st2ed, graph_id, is_bdy, K) -> None:
    """Assert st2ed is a permutation placing each part contiguously in part
    order, boundary vertices first (the sort_and_encode contract)."""
    n = graph_id.shape[0]
    assert sorted(st2ed.tolist()) == list(range(n))
    vn, vo, bn = restate_encode_classes(graph_id, is_bdy, K)
    for p in range(1, K + 1):
        seg = st2ed[vo[p]:vo[p] + vn[p]]
        assert np.all(graph_id[seg] == p)
        assert np.all(is_bdy[seg[:bn[p]]])
        assert not np.any(is_bdy[seg[bn[p]:]])


# --------------------------------------------------------------------------
# The reference binary
# --------------------------------------------------------------------------

def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def run_ref(workdir: str, name: str, directed: bool, weighted: bool, K: int, *,
            parts="all", meta_out: str | None = None, dist_out: str | None = None,
            path_out: str | None = None, rowsum_out: str | None = None,
            threads: int | None = None,
            partition_file: str | None = None, timeout: float | None = None) -> list:
    """Run the reference's CPU path (oracle/_ref/fap_ref) and return its JSON
    event lines."""
    if not ref_available():
        raise FileNotFoundError(REF_BIN)
    cmd = [REF_BIN, "--dir", workdir, "-f", name, "-k", str(K),
           "-direct", str(int(directed)), "-weight", str(int(weighted)),
           "--parts", parts if isinstance(parts, str) else ",".join(map(str, parts))]
    if meta_out:
        cmd += ["--meta", os.path.abspath(meta_out)]
    if dist_out:
        cmd += ["--dist", os.path.abspath(dist_out)]
    if path_out:
        cmd += ["--path", os.path.abspath(path_out)]
    if rowsum_out:
        cmd += ["--rowsum", os.path.abspath(rowsum_out)]
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    if partition_file:
        env["FAP_PARTITION_FILE"] = os.path.abspath(partition_file)
    r = subprocess.run(cmd, check=True, capture_output=True, text=True, env=env,
                       timeout=timeout)
    return [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]


# --------------------------------------------------------------------------
# Comparison helpers
# --------------------------------------------------------------------------

def to_i32(block_f32: np.ndarray) -> np.ndarray:
    """Reference float distances on integer weights -> int32 (exact while the
    finite distances stay below 2^24); the sentinel 1e8 maps to 100000000."""
    return block_f32.astype(np.int64).astype(np.int32)


def row_checksums(block_i32: np.ndarray) -> np.ndarray:
    """Per-row checksum: sum_j uint32(v[j]) * (2j + 1) mod 2^64."""
    b = np.ascontiguousarray(block_i32).view(np.uint32).astype(np.uint64)
    wts = (2 * np.arange(b.shape[1], dtype=np.uint64) + 1)
    with np.errstate(over="ignore"):
        return (b * wts[None, :]).sum(axis=1, dtype=np.uint64)


# --------------------------------------------------------------------------
# Predecessor (path) matrices
# --------------------------------------------------------------------------
#
# The reference records, for every entry, the vertex before j on the
# shortest path it found (path[u] = ver in dijkstra_path,
# fap/kernel/batch_sssp.h:108-110; path[i][j] = path[k][j] in floyd_CPU_path,
# fap/kernel/floyd.h:38-49; path = mat2_path[k][j] for the first minimal k in
# min_plus_path_CPU_advanced, fap/kernel/minplus.h:51-65; edge entries
# path = ver and the diagonal path = the vertex itself in MysubMatBuild_path,
# fap/utils/util_Myalgorithm.h:30-73; -1 where nothing was set).  Which of
# several equally short paths it keeps depends on its evaluation order.  The
# B200 path picks, from the final distances, the in-neighbour u of j with the
# least dist[u] + w(u, j) (the smallest u among equal sums): the same meaning,
# a fixed rule on ties.  port_predecessors restates that rule;
# tests/test_oracle.py pins it to the reference's own matrices on every entry
# whose predecessor is unique.  For the inner rows of parts with few
# boundary vertices the B200 path takes the predecessor off the min-plus
# choice instead (port_predecessors_block), again a valid shortest path that
# agrees wherever the predecessor is unique.

def in_edges(row_offset, col, weight):
    """(tro, tcol, tw): the CSR of in-edges (j's sources in tcol[tro[j]:
    tro[j+1]], ascending), with their weights."""
    ro = np.asarray(row_offset, np.int64)
    n = ro.shape[0] - 1
    m = int(ro[-1])
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(ro))
    dst = np.asarray(col[:m], np.int64)
    w = np.asarray(weight[:m])
    order = np.lexsort((src, dst))
    tro = np.zeros(n + 1, np.int64)
    np.add.at(tro, dst + 1, 1)
    return np.cumsum(tro), src[order], w[order]


def port_predecessors(dist_rows, row_vertices, row_offset, col, weight, integral: bool):
    """P[r][j] = argmin over in-edges (u -> j) of dist_rows[r][u] + w (sums in
    int64 for integer distances, float32 otherwise; the smallest u among
    equal sums), P[r][src] = src, -1 where dist_rows[r][j] >= 1e8."""
    D = np.asarray(dist_rows)
    R, n = D.shape
    tro, tcol, tw = in_edges(row_offset, col, weight)
    if integral:
        Dv = D.astype(np.int64)
        cand = Dv[:, tcol] + tw.astype(np.int64)[None, :]
        big = np.int64(1) << 62
        cand = np.where(Dv[:, tcol] >= 100000000, big, cand)
    else:
        Dv = D.astype(np.float32)
        cand = Dv[:, tcol] + tw.astype(np.float32)[None, :]
        big = np.float32(np.inf)
        cand = np.where(Dv[:, tcol] >= np.float32(1e8), big, cand)
    P = np.full((R, n), -1, np.int64)
    deg = np.diff(tro)
    has = np.nonzero(deg > 0)[0]
    if has.size:
        starts = tro[has]
        mins = np.minimum.reduceat(cand, starts, axis=1)           # (R, |has|)
        seg = np.repeat(np.arange(has.size), deg[has])               # edge -> segment
        at_min = cand == mins[:, seg]
        pos = np.where(at_min, np.arange(tcol.shape[0])[None, :], tcol.shape[0])
        first = np.minimum.reduceat(pos, starts, axis=1)             # first edge with the min
        preds = tcol[np.minimum(first, tcol.shape[0] - 1)]
        ok = mins < big
        P[:, has] = np.where(ok, preds, -1)
    reach = (D < 100000000) if integral else (D.astype(np.float32) < np.float32(1e8))
    P = np.where(reach, P, -1)
    P[np.arange(R), np.asarray(row_vertices)] = np.asarray(row_vertices)
    return P.astype(np.int32)


PRED_THIN_B = 12   # parts with at most this many boundary vertices use the argmin rule


def port_predecessors_block(block, part_vertices, b: int, row_offset, col, weight, integral: bool,
                            thin_b: int = PRED_THIN_B):
    """Predecessor rows of one part's solved block (rows in sorted order:
    the part's b boundary vertices first), as the B200 path produces them:
    boundary rows, own-part columns and parts with more than thin_b boundary
    vertices follow port_predecessors (the in-edge argmin); the inner rows of
    the other parts take, for columns outside the part, the predecessor on
    the row of the boundary vertex k* that the min-plus merge chose -- the
    first k with the least F[i][k] + D[k][j] (F[i][k] = block[i][vertex of
    boundary k], the closed distance the decode wrote) -- or -1 when that
    least sum is the sentinel."""
    D = np.asarray(block)
    verts = np.asarray(part_vertices, np.int64)
    P = port_predecessors(D, verts, row_offset, col, weight, integral).astype(np.int64)
    s, n = D.shape
    if b > thin_b or s <= b:
        return P.astype(np.int32)
    own = np.zeros(n, bool)
    own[verts] = True
    inner = np.arange(b, s)
    if b == 0:
        P[np.ix_(inner, np.nonzero(~own)[0])] = -1
        return P.astype(np.int32)
    if integral:
        A = D[inner][:, verts[:b]].astype(np.int64)
        S = D[:b].astype(np.int64)
        inf = 100000000
    else:
        A = D[inner][:, verts[:b]].astype(np.float32)
        S = D[:b].astype(np.float32)
        inf = np.float32(1e8)
    sums = A[:, :, None] + S[None, :, :]          # inner x b x n
    k_star = np.argmin(sums, axis=1)               # first least k
    best = np.take_along_axis(sums, k_star[:, None, :], axis=1)[:, 0, :]
    Pi = P[:b][k_star, np.arange(n)[None, :]]
    Pi = np.where(best < inf, Pi, -1)
    cols = np.nonzero(~own)[0]
    P[np.ix_(inner, cols)] = Pi[:, cols]
    return P.astype(np.int32)


def port_predecessors_parts(dist_sorted, st2ed, ver_num, ver_offset, bdy_num, row_offset, col, weight,
                            integral: bool, thin_b: int = PRED_THIN_B):
    """port_predecessors_block over every part of a full n x n matrix in
    sorted row order."""
    D = np.asarray(dist_sorted)
    out = np.empty(D.shape, np.int32)
    for p in range(1, len(ver_num)):
        off, s = int(ver_offset[p]), int(ver_num[p])
        if s == 0:
            continue
        out[off:off + s] = port_predecessors_block(D[off:off + s], st2ed[off:off + s], int(bdy_num[p]),
                                                   row_offset, col, weight, integral, thin_b)
    return out


def unique_predecessor_mask(dist_rows, row_vertices, row_offset, col, weight, integral: bool,
                            rel_gap: float = 1e-5):
    """Entries whose best in-edge is strictly better than the second best (by
    rel_gap for float sums) and consistent with dist_rows[r][j]: there, every
    shortest-path order must pick the same predecessor."""
    D = np.asarray(dist_rows)
    R, n = D.shape
    tro, tcol, tw = in_edges(row_offset, col, weight)
    Dv = D.astype(np.float64)
    cand = Dv[:, tcol] + np.asarray(tw, np.float64)[None, :]
    cand = np.where(Dv[:, tcol] >= 1e8, np.inf, cand)
    out = np.zeros((R, n), bool)
    for j in range(n):
        a, b = tro[j], tro[j + 1]
        if b - a == 0:
            continue
        c = np.sort(cand[:, a:b], axis=1)
        best = c[:, 0]
        second = c[:, 1] if b - a > 1 else np.full(R, np.inf)
        # distinct in-neighbours only: duplicates of the best edge make ties
        srcs = tcol[a:b]
        if len(np.unique(srcs)) != len(srcs):
            continue
        with np.errstate(invalid="ignore"):
            gap = (second - best) > (0.0 if integral else rel_gap * np.maximum(best, 1e-30))
        consistent = np.abs(best - Dv[:, j]) <= (0.0 if integral else 1e-5 * np.maximum(Dv[:, j], 1e-30))
        out[:, j] = gap & consistent & (Dv[:, j] < 1e8)
    out[np.arange(R), np.asarray(row_vertices)] = False
    return out


def check_paths(dist_rows, pred_rows, row_vertices, row_offset, col, weight, integral: bool,
                rel_tol: float = 1e-5):
    """Validity of predecessor rows: the source maps to itself, unreachable
    entries are -1, every other entry names an in-neighbour u of j with
    dist[u] + w(u, j) == dist[j] (within rel_tol for float), and following
    predecessors from any reachable vertex ends at the source.  Returns the
    number of entries checked; raises AssertionError on the first failure."""
    D = np.asarray(dist_rows, np.float64)
    P = np.asarray(pred_rows, np.int64)
    R, n = D.shape
    ro = np.asarray(row_offset, np.int64)
    m = int(ro[-1])
    wmin = {}
    for u in range(n):
        for e in range(ro[u], ro[u + 1]):
            key = (u, int(col[e]))
            wmin[key] = min(wmin.get(key, np.inf), float(weight[e]))
    checked = 0
    for r in range(R):
        s = int(row_vertices[r])
        assert P[r, s] == s, f"row {r}: source {s} maps to {P[r, s]}"
        reach = D[r] < 1e8
        assert np.all(P[r, ~reach] == -1), f"row {r}: unreachable entries with predecessors"
        for j in np.nonzero(reach)[0]:
            if j == s:
                continue
            u = int(P[r, j])
            assert (u, int(j)) in wmin, f"row {r}: {u} -> {j} is not an edge"
            got = D[r, u] + wmin[(u, int(j))]
            tol = 0.0 if integral else rel_tol * max(abs(D[r, j]), 1e-30)
            assert abs(got - D[r, j]) <= tol, f"row {r}: d[{u}] + w = {got} != d[{j}] = {D[r, j]}"
            checked += 1
        # pointer doubling: every reachable vertex must lead to the source
        Q = np.where(reach, P[r], s)
        for _ in range(int(np.ceil(np.log2(max(n, 2)))) + 1):
            Q = Q[Q]
        assert np.all(Q[reach] == s), f"row {r}: predecessor chain does not reach the source"
    return checked
