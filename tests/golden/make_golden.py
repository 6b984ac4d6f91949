"""Generates the golden fixtures in this directory from the reference itself.

Run in a container that has the reference sources (oracle/_ref/fap_ref is
built from them by `make -C oracle ref`):

    python tests/golden/make_golden.py

Each case is a small seeded graph written as MatrixMarket; the reference's
CPU path (fapGraph::run per part, driven by oracle/_ref/fap_ref) solves it
and the fixture stores the graph text, the reference's partition and
renumbering, and its distances (full matrix for small cases, per-row
checksums plus sampled rows for the 64x64 grid) and, for the full cases,
its predecessor matrix (row i, column j: the vertex before j on the
reference's shortest path from row i's vertex; -1 unreachable).  Directed cases use a
given contiguous partition (FAP_PARTITION_FILE), because the reference's
METIS input for directed graphs is misaligned when a vertex has no edge.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fastapsp_b200 import generators as G  # noqa: E402
from oracle import oracle as O  # noqa: E402


def road_with_quirks(n, seed):
    g = G.road_graph(n, seed=seed)
    rng = np.random.default_rng(seed + 100)
    # duplicate edges with other weights, and self-loops
    dup = g.edges[rng.choice(g.edges.shape[0], 6, replace=False)]
    loops = np.stack([rng.integers(0, n, 2)] * 2, 1)
    e = np.concatenate([g.edges, dup, loops], 0)
    w = np.concatenate([g.weights, rng.integers(1, 1001, 8).astype(np.float32)])
    g.edges, g.weights = e, w
    return g


def disconnected():
    a = G.grid_graph(6, 6, seed=5)
    b = G.grid_graph(5, 7, seed=6)
    n = a.n + b.n + 4  # four isolated vertices
    e = np.concatenate([a.edges, b.edges + a.n], 0)
    return G.EdgeList(n, e, np.ones(e.shape[0], np.float32), directed=False, weighted=False,
                      integral=True, info={"kind": "disconnected"})


def rgg_float(n, seed):
    """Duplicate-free random geometric graph with float weights: shortest
    paths are unique with probability one, so predecessors compare exactly."""
    g = G.road_graph(n, seed=seed, target_avg_degree=2.6)
    rng = np.random.default_rng(seed + 7)
    g.weights = rng.uniform(0.5, 100.0, g.edges.shape[0]).astype(np.float32)
    g.integral = False
    return g


def rmat_int(scale, m, seed):
    g = G.rmat_graph(scale, m, seed=seed)
    rng = np.random.default_rng(seed)
    g.weights = rng.integers(1, 101, g.edges.shape[0]).astype(np.float32)
    g.integral = True
    return g


CASES = {
    # name: (maker, K, partition: None = METIS, "contig" = contiguous ranges, full dist?)
    "grid12_k4": (lambda: G.grid_graph(12, 12, drop_frac=0.05, seed=11), 4, None, True),
    "road300_k6": (lambda: road_with_quirks(300, 12), 6, None, True),
    "disconnected_k3": (disconnected, 3, None, True),
    # K=1: the reference's METIS call dies with SIGFPE for one part, so the
    # (trivial) partition is given
    "grid10_k1": (lambda: G.grid_graph(10, 10, seed=13, wmin=1, wmax=9), 1, "contig", True),
    "rmat8_int_k4": (lambda: rmat_int(8, 2048, 14), 4, "contig", True),
    "rmat8_f32_k4": (lambda: G.rmat_graph(8, 2048, seed=15), 4, "contig", True),
    "rgg300_f32_k4": (lambda: rgg_float(300, 16), 4, None, True),
    "grid64_k8": (lambda: G.grid_graph(64, 64, drop_frac=0.02, seed=1), 8, None, False),
}


def make_case(name, maker, K, partition, full, tmp):
    g = maker()
    root = os.path.join(tmp, name)
    path = G.write_mtx(g, root, name)
    mtx_text = open(path).read()
    part_file = None
    gid0 = None
    if partition == "contig":
        gid0 = (np.arange(g.n, dtype=np.int64) * K // g.n).astype(np.int32)
        part_file = os.path.join(tmp, name + ".part")
        gid0.tofile(part_file)
    meta_f = os.path.join(tmp, name + ".meta")
    dist_f = os.path.join(tmp, name + ".dist")
    path_f = os.path.join(tmp, name + ".path")
    ev = O.run_ref(root, name, g.directed, g.weighted, K, meta_out=meta_f, dist_out=dist_f,
                   path_out=path_f if full else None, partition_file=part_file)
    meta = O.read_meta(meta_f)
    dist = np.fromfile(dist_f, dtype=np.float32).reshape(meta.n, meta.n)
    out = dict(name=name, mtx=np.array(mtx_text), directed=g.directed, weighted=g.weighted,
               integral=g.integral, K=K, n=meta.n, m=meta.m,
               row_offset=meta.row_offset, col_val=meta.col_val, weight=meta.weight,
               graph_id=meta.graph_id, st2ed=meta.st2ed, ver_num=meta.ver_num,
               ver_offset=meta.ver_offset, bdy_num=meta.bdy_num,
               injected_partition=np.array(partition is not None))
    if full:
        out["dist"] = dist
        out["path"] = np.fromfile(path_f, dtype=np.int32).reshape(meta.n, meta.n)
    else:
        out["row_checksums"] = O.row_checksums(O.to_i32(dist))
        rng = np.random.default_rng(0)
        rows = np.sort(rng.choice(meta.n, 16, replace=False))
        out["sample_rows"] = rows
        out["sample_dist"] = dist[rows]
    if g.integral:
        fin = dist[dist < 1e8]
        assert fin.size == 0 or fin.max() < 2 ** 24, "int32 parity needs distances < 2^24"
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "n", meta.n, "K", K, "bdy", meta.bdy_num[1:].tolist(), "parts", len(ev) - 1)


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/fap_ref missing: run `make -C oracle ref` first")
    with tempfile.TemporaryDirectory() as tmp:
        for name, (maker, K, part, full) in CASES.items():
            make_case(name, maker, K, part, full, tmp)


if __name__ == "__main__":
    main()
