"""Seeded synthetic graphs of the shapes the APSP benchmarks are quoted on,
and a MatrixMarket writer in the layout the fapGraph reader consumes.

Edges are returned as an (E, 2) int64 array of 0-based endpoints plus an (E,)
weight array.  For undirected graphs each undirected edge appears once; the
reader inserts both directions (fap/utils/readMatFile.h:112-128).

The reader takes |w| as float32 (fap/utils/readMatFile.h:124-125,140-141), so
float weights are written with 9 significant digits, which round-trips every
float32 exactly.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class EdgeList:
    n: int
    edges: np.ndarray          # (E, 2) int64, 0-based
    weights: np.ndarray        # (E,) float32 (integral values for int weights)
    directed: bool
    weighted: bool
    integral: bool             # weights are integers (int32 compute path)
    info: dict = field(default_factory=dict)

    @property
    def num_input_edges(self) -> int:
        return int(self.edges.shape[0])


def kind_dir(directed: bool, weighted: bool) -> str:
    """Sub-directory name the reference resolves (readMatFile.h:43-51)."""
    return ("weight" if weighted else "unweight") + "-" + (
        "directed" if directed else "undirected")


def mtx_path(root: str, name: str, directed: bool, weighted: bool) -> str:
    return os.path.join(root, "graph", kind_dir(directed, weighted), name + ".mtx")


def write_mtx(g: EdgeList, root: str, name: str) -> str:
    """Write g as root/graph/<kind>/<name>.mtx: header 'n n m' then one
    1-based 'a b [w]' line per input edge."""
    path = mtx_path(root, name, g.directed, g.weighted)
    os.makedirs(os.path.dirname(path), exist_ok=True)
    a = g.edges[:, 0] + 1
    b = g.edges[:, 1] + 1
    with open(path, "w") as f:
        f.write(f"{g.n} {g.n} {g.num_input_edges}\n")
        if not g.weighted:
            np.savetxt(f, np.stack([a, b], 1), fmt="%d")
        elif g.integral:
            np.savetxt(f, np.stack([a, b, g.weights.astype(np.int64)], 1), fmt="%d")
        else:
            lines = "".join(f"{x} {y} {float(w):.9g}\n"
                            for x, y, w in zip(a.tolist(), b.tolist(), g.weights.tolist()))
            f.write(lines)
    return path


# --------------------------------------------------------------------------
# Generators
# --------------------------------------------------------------------------

def grid_graph(rows: int, cols: int, *, drop_frac: float = 0.0, extra_frac: float = 0.0,
               wmin: int = 1, wmax: int = 1, seed: int = 0) -> EdgeList:
    """4-neighbour rows x cols grid, a fraction of its edges dropped uniformly
    at random, plus extra_frac x (grid edges) random long-range edges.
    Unit weights when wmin == wmax == 1 (unweighted MTX), else integer weights
    uniform in [wmin, wmax]."""
    rng = np.random.default_rng(seed)
    idx = np.arange(rows * cols, dtype=np.int64).reshape(rows, cols)
    h = np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], 1)
    v = np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()], 1)
    e = np.concatenate([h, v], 0)
    base = e.shape[0]
    if drop_frac > 0:
        keep = rng.random(base) >= drop_frac
        e = e[keep]
    n = rows * cols
    if extra_frac > 0:
        k = int(round(extra_frac * base))
        a = rng.integers(0, n, size=2 * k)
        b = rng.integers(0, n, size=2 * k)
        ok = a != b
        x = np.stack([a[ok], b[ok]], 1)
        # drop pairs that duplicate an existing edge (either orientation)
        seen = set(map(tuple, np.sort(e, 1).tolist()))
        extra = []
        for p in np.sort(x, 1).tolist():
            t = tuple(p)
            if t not in seen:
                seen.add(t)
                extra.append(p)
            if len(extra) == k:
                break
        e = np.concatenate([e, np.asarray(extra, dtype=np.int64).reshape(-1, 2)], 0)
    weighted = not (wmin == 1 and wmax == 1)
    w = (rng.integers(wmin, wmax + 1, size=e.shape[0]).astype(np.float32)
         if weighted else np.ones(e.shape[0], np.float32))
    return EdgeList(n, e, w, directed=False, weighted=weighted, integral=True,
                    info={"kind": "grid", "rows": rows, "cols": cols,
                          "drop_frac": drop_frac, "extra_frac": extra_frac,
                          "seed": seed, "grid_edges": base})


def road_graph(n: int, *, seed: int = 0, wmin: int = 1, wmax: int = 1000,
               target_avg_degree: float = 2.1) -> EdgeList:
    """Road-network-shaped graph: n points uniform in the unit square; the
    Euclidean minimum spanning tree (every vertex joined to a near neighbour,
    near-planar, large hop diameter) plus extra nearest-neighbour edges (each
    vertex's 2nd/3rd nearest) until the average degree reaches
    target_avg_degree.  Integer weights uniform in [wmin, wmax]."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import minimum_spanning_tree
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    tree = cKDTree(pts)
    dist, nbr = tree.query(pts, k=4)              # self + 3 nearest
    src = np.repeat(np.arange(n), 3)
    dst = nbr[:, 1:].ravel()
    d = dist[:, 1:].ravel()
    # Candidate graph = 3-NN graph; its MST may be a forest, so join the
    # components with the Delaunay graph edges as well.
    from scipy.spatial import Delaunay
    tri = Delaunay(pts)
    s = tri.simplices
    de = np.concatenate([s[:, [0, 1]], s[:, [1, 2]], s[:, [0, 2]]], 0)
    dd = np.linalg.norm(pts[de[:, 0]] - pts[de[:, 1]], axis=1)
    ca = np.concatenate([src, de[:, 0]])
    cb = np.concatenate([dst, de[:, 1]])
    cd = np.concatenate([d, dd]) + 1e-12
    lo = np.minimum(ca, cb)
    hi = np.maximum(ca, cb)
    g = coo_matrix((cd, (lo, hi)), shape=(n, n)).tocsr()
    g.sum_duplicates()
    mst = minimum_spanning_tree(g).tocoo()
    tree_e = np.stack([mst.row, mst.col], 1).astype(np.int64)
    tree_set = set(map(tuple, np.sort(tree_e, 1).tolist()))
    target_m = int(round(target_avg_degree * n / 2))
    need = max(0, target_m - tree_e.shape[0])
    # extra edges: random vertices joined to their 2nd or 3rd nearest neighbour
    order = rng.permutation(n)
    extra = []
    for u in order.tolist():
        if len(extra) >= need:
            break
        v = int(nbr[u, 1 + int(rng.integers(1, 3))])
        t = (min(u, v), max(u, v))
        if u != v and t not in tree_set:
            tree_set.add(t)
            extra.append(t)
    e = np.concatenate([tree_e, np.asarray(extra, np.int64).reshape(-1, 2)], 0)
    e = e[rng.permutation(e.shape[0])]
    w = rng.integers(wmin, wmax + 1, size=e.shape[0]).astype(np.float32)
    return EdgeList(n, e, w, directed=False, weighted=True, integral=True,
                    info={"kind": "road", "n": n, "seed": seed,
                          "avg_degree": 2.0 * e.shape[0] / n,
                          "tree_edges": int(tree_e.shape[0]), "extra_edges": len(extra)})


def rmat_graph(scale: int, num_edges: int, *, a=0.57, b=0.19, c=0.19, seed: int = 0,
               wlo: float = 0.01, whi: float = 100.0) -> EdgeList:
    """Directed R-MAT graph on 2^scale vertices: num_edges edges drawn with
    quadrant probabilities (a, b, c, 1-a-b-c); self-loops dropped, duplicate
    edges kept (the CSR keeps every input line).  float32 weights
    log-uniform in [wlo, whi]."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    src = np.zeros(num_edges, np.int64)
    dst = np.zeros(num_edges, np.int64)
    for bit in range(scale):
        r = rng.random(num_edges)
        right = (r >= a) & (r < a + b) | (r >= a + b + c)
        down = r >= a + b
        src |= down.astype(np.int64) << bit
        dst |= right.astype(np.int64) << bit
    keep = src != dst
    e = np.stack([src[keep], dst[keep]], 1)
    w = np.exp(rng.uniform(np.log(wlo), np.log(whi), size=e.shape[0])).astype(np.float32)
    return EdgeList(n, e, w, directed=True, weighted=True, integral=False,
                    info={"kind": "rmat", "scale": scale, "edges_drawn": num_edges,
                          "self_loops_dropped": int((~keep).sum()), "seed": seed})


def random_geometric_graph(n: int, avg_degree: float, *, seed: int = 0,
                           wmin: int = 1, wmax: int = 1000) -> EdgeList:
    """Connected random geometric graph (EMST backbone plus nearest-neighbour
    edges up to avg_degree) with integer weights; used by the serving stream."""
    return road_graph(n, seed=seed, wmin=wmin, wmax=wmax, target_avg_degree=avg_degree)


def edges_to_csr(g: EdgeList):
    """CSR (row_offset, col_val, weight) of g with both directions of every
    undirected edge; within a row, edges keep their input order."""
    e = g.edges
    if g.directed:
        src, dst, w = e[:, 0], e[:, 1], g.weights
    else:
        src = np.concatenate([e[:, 0], e[:, 1]])
        dst = np.concatenate([e[:, 1], e[:, 0]])
        w = np.concatenate([g.weights, g.weights])
    order = np.argsort(src, kind="stable")
    ro = np.zeros(g.n + 1, np.int64)
    np.add.at(ro, src + 1, 1)
    return (np.cumsum(ro).astype(np.int32), dst[order].astype(np.int32),
            w[order].astype(np.float32))


# --------------------------------------------------------------------------
# The serving stream: many resident graphs of different sizes
# --------------------------------------------------------------------------

def serve_specs(count: int = 32, seed: int = 17, n_range=(16000, 200000),
                rows_range=(100, 10000), degree_range=(2.0, 4.0)) -> list:
    """Seeded specs of the serving stream's random-geometric graphs: n
    log-uniform in n_range, average degree uniform in degree_range, int
    weights U[1,1000], and K a power of two in [16, 256] chosen so that the
    parts' row counts (n / K) spread log-uniformly over rows_range."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        rows = np.exp(rng.uniform(np.log(rows_range[0]), np.log(rows_range[1])))
        K = int(2 ** np.clip(np.round(np.log2(n / rows)), 4, 8))
        specs.append(dict(name=f"rgg{i:02d}", n=n, K=K,
                          avg_degree=float(rng.uniform(*degree_range)), seed=1000 + i))
    return specs


def serve_graph_csr(spec: dict):
    """(spec, row_offset, col_val, weight) of one serving-stream graph
    (module-level so that a process pool can build the graphs in parallel)."""
    el = random_geometric_graph(spec["n"], spec["avg_degree"], seed=spec["seed"])
    return (spec,) + edges_to_csr(el)


# --------------------------------------------------------------------------
# The benchmark workloads, by name
# --------------------------------------------------------------------------

WORKLOADS = {
    # 64x64 grid, 2% of edges dropped, unit weights, K=8
    "grid64": dict(make=lambda: grid_graph(64, 64, drop_frac=0.02, seed=1), K=8),
    # 114,599-vertex road-shaped graph, int weights in [1,1000], K=128
    "road114k": dict(make=lambda: road_graph(114599, seed=2), K=128),
    # profiling-size stand-in for road114k: same part size (~830 vertices)
    "road20k": dict(make=lambda: road_graph(20000, seed=9), K=24),
    # 512x512 grid + 1% long-range edges, int weights in [1,100], K=256
    "grid512": dict(make=lambda: grid_graph(512, 512, extra_frac=0.01, wmin=1, wmax=100,
                                            seed=3), K=256),
    # min-plus profiling case of the grid shape: ~1024-vertex parts with
    # ~120 boundary vertices, 1 GB of output
    "grid128": dict(make=lambda: grid_graph(128, 128, extra_frac=0.01, wmin=1, wmax=100,
                                            seed=7), K=16),
    # profiling-size stand-in for grid512: same part size (~1024 vertices),
    # over 8192 boundary vertices (the Bellman-Ford closure of the boundary graph)
    "grid256": dict(make=lambda: grid_graph(256, 256, extra_frac=0.01, wmin=1, wmax=100,
                                            seed=5), K=64),
    # profiling-size stand-in for rmat16: same average degree and part size
    "rmat14": dict(make=lambda: rmat_graph(14, 1 << 18, seed=6), K=16),
    # R-MAT scale 16, 2^20 directed edges, float weights, K=64
    "rmat16": dict(make=lambda: rmat_graph(16, 1 << 20, seed=4), K=64),
}
