"""Benchmark workloads: seeded synthetic graphs of the named shapes, written
as MatrixMarket and loaded through the drop-in fapGraph (host IO, METIS,
boundary detection and renumbering).

`write()` only generates the graph and writes its MatrixMarket file; it
neither imports the fapGraph binding nor loads libfap_b200.so, so a process
that drives the reference's own binary on that file (the reference arm of
the benchmark) runs none of this library's code."""
from __future__ import annotations

import os
import tempfile
from dataclasses import dataclass

import numpy as np

from . import generators as G


@dataclass
class Workload:
    name: str
    K: int
    edges: G.EdgeList
    root: str           # directory holding graph/<kind>/<name>.mtx
    graph: "fapGraph"   # after preCondition
    n: int
    ver_num: np.ndarray
    ver_offset: np.ndarray
    bdy_num: np.ndarray

    @property
    def entries(self) -> int:
        return self.n * self.n

    def csr(self):
        return self.graph.csr()

    def data_description(self) -> str:
        info = self.edges.info
        kind = info.get("kind")
        if kind == "road":
            return ("synthetic: seeded road-shaped graph (uniform points, Euclidean MST + "
                    "nearest-neighbour edges), int weights U[1,1000]")
        if kind == "grid":
            return (f"synthetic: seeded {info['rows']}x{info['cols']} grid, "
                    f"{info['drop_frac']:.0%} edges dropped, {info['extra_frac']:.0%} extra random "
                    "edges, int weights")
        if kind == "rmat":
            return ("synthetic: seeded directed R-MAT (0.57, 0.19, 0.19, 0.05), self-loops dropped, "
                    "duplicates kept, float weights log-uniform [0.01, 100]")
        return "synthetic"

    def describe(self) -> dict:
        vn, bn = self.ver_num[1:], self.bdy_num[1:]
        return {"workload": self.name, "n": self.n, "arcs": int(self.graph.csr()[0][-1]),
                "K": self.K, "directed": self.edges.directed,
                "avg_degree": round(float(self.graph.csr()[0][-1]) / self.n, 3),
                "part_size": [int(vn.min()), int(np.median(vn)), int(vn.max())],
                "boundary": [int(bn.min()), int(np.median(bn)), int(bn.max()), int(bn.sum())]}


@dataclass
class WorkloadFile:
    """A workload's MatrixMarket file on disk (no partition, no library)."""
    name: str
    K: int
    edges: G.EdgeList
    root: str           # directory holding graph/<kind>/<name>.mtx

    @property
    def n(self) -> int:
        return self.edges.n


def write(name: str, root: str | None = None) -> WorkloadFile:
    """Generates workload `name` (seeded) and writes its MatrixMarket file
    under root/graph/<kind>/ in the layout the reference's reader resolves."""
    spec = G.WORKLOADS[name]
    el = spec["make"]()
    root = root or tempfile.mkdtemp(prefix="fap_wl_")
    path = G.mtx_path(root, name, el.directed, el.weighted)
    if not os.path.exists(path):
        G.write_mtx(el, root, name)
    return WorkloadFile(name, spec["K"], el, root)


def load(name: str, root: str | None = None) -> Workload:
    from .graph import fapGraph
    wf = write(name, root)
    el, root = wf.edges, wf.root
    spec = G.WORKLOADS[name]
    g = fapGraph(name, el.directed, el.weighted, spec["K"], root=root)
    g.preCondition()
    vn, vo, bn = g.partInfo()
    return Workload(name, spec["K"], el, root, g, g.num_vertexs, vn, vo, bn)


@dataclass
class ServeGraph:
    name: str
    n: int
    K: int
    avg_degree: float
    graph: "fapGraph"   # after preCondition (partition + renumbering)


def load_serve_stream(count: int = 32, procs: int = 0, seed: int = 17) -> list:
    """The serving stream's resident graphs (generators.serve_specs), built in
    a spawn-started process pool and partitioned on the host (METIS)."""
    import multiprocessing as mp

    from .graph import fapGraph
    specs = G.serve_specs(count, seed)
    procs = procs or max(1, min(8, os.cpu_count() or 1, count))
    if procs > 1:
        with mp.get_context("spawn").Pool(procs) as pool:
            built = pool.map(G.serve_graph_csr, specs)
    else:
        built = [G.serve_graph_csr(s) for s in specs]
    out = []
    for spec, ro, col, w in built:
        g = fapGraph.from_csr(spec["n"], int(ro[-1]), ro, col, w, spec["K"])
        g.preCondition()
        out.append(ServeGraph(spec["name"], spec["n"], spec["K"],
                              round(float(ro[-1]) / spec["n"], 3), g))
    return out
